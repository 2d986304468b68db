// layout.cpp -- host builder of the reference's device buffer layout.
//
// Restates, for a flat synapse list, what Simulation's constructor builds
// (Simulation.ipp:108-118):
//   NeuronData::initialize     NeuronData.ipp:27-170   SoA [(k*P + p)*MPS + n]
//   SynapseData::initialize    SynapseData.ipp:8-111   bundles of BUNDLE_SIZE slots,
//                                                      bundle 0 unused, delay bitmap
//   SynapseIndex::addSynapse   SynapseIndex.cpp:42-63
//   GroupData::initialize      GroupData.cpp:70-228    groupPtrs / groupMatrix,
//                                                      pitch, step, max incoming bundles
//   GlobalQueue / LocalQueue / SpikeBuffer / CurrentData ::initialize (sizes)
// Differences, each a superset of the reference's buffers: the global-queue
// counters and rows, and firedOutput, are sized for all partitions (the
// reference sizes them for neuron partitions only, GlobalQueue.cpp:22,32 and
// SpikeBuffer.cpp:86, while gather/scatter and the input kernel index them for
// every partition).  Source keys are visited in ascending (partition, neuron,
// delay) order and target partitions ascending; the reference walks
// boost::unordered_map order, which only permutes rows of groupMatrix.
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/szsnn_cuda.h"

struct szsnn_layout {
    szsnn_layout_consts c{};
    szsnn_layout_info info{};
    std::vector<uint32_t> partition_sizes;
    std::vector<float> nparams, nvars, iparams, ivars;
    std::vector<uint32_t> targets;
    std::vector<float> weights;
    std::vector<uint64_t> delay_bits;
    std::vector<uint32_t> group_ptrs;    // uint2 pairs
    std::vector<uint32_t> group_matrix;  // uint2 pairs
};

namespace {

uint64_t align_up(uint64_t a, uint64_t b) { return b * ((a + b - 1) / b); }

uint32_t ceil_pow2(uint32_t val)  // GroupData.cpp:58-68, unsigned wrap for 0 included
{
    val--;
    val |= val >> 1;
    val |= val >> 2;
    val |= val >> 4;
    val |= val >> 8;
    val |= val >> 16;
    val++;
    return val;
}

int fail(char* err, size_t len, int code, const std::string& m)
{
    if (err && len) {
        std::strncpy(err, m.c_str(), len - 1);
        err[len - 1] = 0;
    }
    return code;
}

}  // namespace

extern "C" int szsnn_layout_build(const szsnn_layout_consts* consts, const szsnn_layout_desc* d,
                                  szsnn_layout** out, char* err, size_t err_len)
{
    if (!consts || !d || !out) return fail(err, err_len, SZSNN_ERR_ARG, "null argument");
    *out = nullptr;
    const uint64_t MPS = consts->max_partition_size, B = consts->warp_size, D = consts->max_synaptic_delay;
    const uint64_t TPG = consts->threads_per_group;
    if (MPS == 0 || MPS > 1024 || MPS % 32 || B == 0 || B > 32 || D == 0 || D > 64 || TPG == 0)
        return fail(err, err_len, SZSNN_ERR_ARG, "bad layout constants");
    if (d->n_neurons == 0) return fail(err, err_len, SZSNN_ERR_ARG, "network has 0 neurons");  // Simulation.ipp:97-101
    if (d->n_inputs > MPS)
        return fail(err, err_len, SZSNN_ERR_LIMIT, "more inputs than MAX_INPUTS_SIZE");  // NetworkGraph.ipp:454-458
    if (d->add_phony_synapse && D < 2)
        return fail(err, err_len, SZSNN_ERR_LIMIT, "phony synapse needs MAX_SYNAPTIC_DELAY >= 2");

    szsnn_layout* L = new szsnn_layout();
    L->c = *consts;
    const uint64_t Pn = (d->n_neurons - 1) / MPS + 1;
    const uint64_t Pin = d->n_inputs ? 1 : 0;
    const uint64_t Pt = Pn + Pin;
    const uint64_t bvwp = MPS / 32;
    const uint64_t input_base = Pn * MPS;
    L->info.neuron_partitions = (uint32_t)Pn;
    L->info.input_partitions = (uint32_t)Pin;
    L->info.total_partitions = (uint32_t)Pt;

    // partition sizes (NetworkGraph.ipp:87-93 + input partition)
    L->partition_sizes.assign(Pt, (uint32_t)MPS);
    L->partition_sizes[Pn - 1] = (uint32_t)((d->n_neurons - 1) % MPS + 1);
    if (Pin) L->partition_sizes[Pn] = d->n_inputs;

    // NeuronData SoA
    auto soa = [&](std::vector<float>& dst, uint32_t count, uint64_t parts, const float* src, uint32_t n) {
        dst.assign((size_t)count * parts * MPS, 0.0f);
        if (!src) return;
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t k = 0; k < count; ++k)
                dst[((uint64_t)k * parts + i / MPS) * MPS + i % MPS] = src[(uint64_t)i * count + k];
    };
    soa(L->nparams, d->neuron_param_count, Pn, d->neuron_params, d->n_neurons);
    soa(L->nvars, d->neuron_var_count, Pn, d->neuron_vars, d->n_neurons);
    if (Pin) {
        soa(L->iparams, d->input_param_count, 1, d->input_params, d->n_inputs);
        soa(L->ivars, d->input_var_count, 1, d->input_vars, d->n_inputs);
    }

    // synapse list in the order SynapseData walks it: by source id, insertion
    // order within a source, the phony synapse last among source 0's
    struct Syn { uint32_t s, t; float w; uint32_t d1; };
    std::vector<Syn> syn;
    syn.reserve(d->n_synapses + 1);
    for (uint64_t i = 0; i < d->n_synapses; ++i) {
        Syn s{d->src[i], d->tgt[i], d->weight[i], d->delay1[i]};
        bool src_ok = s.s < d->n_neurons || (s.s >= input_base && s.s < input_base + d->n_inputs);
        if (!src_ok || s.t >= d->n_neurons) {
            delete L;
            return fail(err, err_len, SZSNN_ERR_ARG, "synapse " + std::to_string(i) + " connects nonexisting neurons");
        }
        if (s.d1 < 1 || s.d1 > D) {
            delete L;
            return fail(err, err_len, SZSNN_ERR_LIMIT,
                        "synapse " + std::to_string(i) + " delay outside 1..MAX_SYNAPTIC_DELAY");
        }
        syn.push_back(s);
    }
    if (d->add_phony_synapse) syn.push_back(Syn{0, 0, 0.0f, 2});
    std::stable_sort(syn.begin(), syn.end(), [](const Syn& a, const Syn& b) { return a.s < b.s; });

    // SynapseIndex + SynapseData::addSynapse
    typedef std::tuple<uint32_t, uint32_t, uint32_t, uint32_t> gkey;  // p, n, tp, d1
    typedef std::tuple<uint32_t, uint32_t, uint32_t> skey;            // p, n, d1
    std::map<gkey, uint32_t> group_count;
    std::map<skey, std::map<uint32_t, std::vector<uint32_t>>> bundles;
    std::map<skey, uint32_t> source_count;
    uint64_t next_free = 1;
    L->targets.assign(next_free * B, 0);
    L->weights.assign(next_free * B, 0.0f);
    for (const Syn& s : syn) {
        uint32_t p = (uint32_t)(s.s / MPS), n = (uint32_t)(s.s % MPS);
        uint32_t tp = (uint32_t)(s.t / MPS), tn = (uint32_t)(s.t % MPS);
        uint32_t& gc = group_count[gkey(p, n, tp, s.d1)];
        uint32_t idx = (uint32_t)(gc % B);
        gc += 1;
        std::vector<uint32_t>& vec = bundles[skey(p, n, s.d1)][tp];
        uint64_t row;
        if (idx == 0) {
            vec.push_back((uint32_t)next_free);
            source_count[skey(p, n, s.d1)] += 1;
            row = next_free;
            next_free += 1;
            L->targets.resize(next_free * B, 0);
            L->weights.resize(next_free * B, 0.0f);
        } else {
            row = vec.back();
        }
        L->targets[row * B + idx] = tn;
        L->weights[row * B + idx] = s.w;
    }
    L->info.bundles = next_free;

    // delay bitmap (SynapseData.ipp:53-84): one uint64 per source neuron
    const uint64_t net_size = Pin ? (MPS * Pn + d->n_inputs) : d->n_neurons;
    L->delay_bits.assign(net_size, 0);
    for (auto& kv : bundles) {
        uint32_t p = std::get<0>(kv.first), n = std::get<1>(kv.first), d1 = std::get<2>(kv.first);
        L->delay_bits[(uint64_t)p * MPS + n] |= (uint64_t)1 << (d1 - 1);
    }

    // GroupData (GroupData.cpp:94-228)
    L->group_ptrs.assign(Pt * MPS * D * 2, 0);
    std::map<uint32_t, uint64_t> incoming;
    uint64_t words = 0;
    uint32_t max_bundles_per_nd = 0;
    for (auto& kv : bundles) {
        uint32_t p = std::get<0>(kv.first), n = std::get<1>(kv.first), d1 = std::get<2>(kv.first);
        uint32_t src_count = source_count[kv.first];
        uint32_t wc = (uint32_t)align_up(src_count, B);
        max_bundles_per_nd = std::max(max_bundles_per_nd, wc);
        L->group_matrix.resize((words + wc) * 2, 0);
        uint64_t row_begin = words, col = 0;
        for (auto& tv : kv.second) {
            incoming[tv.first] += tv.second.size();
            for (uint32_t b : tv.second) {
                L->group_matrix[(row_begin + col) * 2 + 0] = tv.first;
                L->group_matrix[(row_begin + col) * 2 + 1] = b;
                ++col;
            }
        }
        uint64_t addr = ((uint64_t)p * MPS + n) * D + (d1 - 1);  // GROUP_ADDR_OFFSET (types.h:113-114)
        L->group_ptrs[addr * 2 + 0] = (uint32_t)row_begin;
        L->group_ptrs[addr * 2 + 1] = (uint32_t)col;
        words += wc;
    }
    uint64_t max_incoming = 0;
    for (auto& kv : incoming) max_incoming = std::max(max_incoming, kv.second);
    uint32_t pitch = std::max(1u, ceil_pow2(max_bundles_per_nd));
    if (pitch > TPG) {
        delete L;
        return fail(err, err_len, SZSNN_ERR_LIMIT,
                    "pitch > THREADS_PER_GROUP (" + std::to_string(pitch) + " > " + std::to_string(TPG) + ")");
    }
    uint32_t step = (uint32_t)(TPG / pitch);
    if ((uint64_t)step * pitch != TPG) {
        delete L;
        return fail(err, err_len, SZSNN_ERR_LIMIT, "step * pitch != THREADS_PER_GROUP");
    }
    L->info.group_pitch = pitch;
    L->info.group_step = step;
    L->info.gq_pitch = max_incoming;

    const uint64_t lq_width = align_up(MPS * D, 32);
    uint64_t* by = L->info.bytes;
    by[SZSNN_L_PARTITION_SIZES] = Pt * 4;
    by[SZSNN_L_NEURON_PARAMS] = L->nparams.size() * 4;
    by[SZSNN_L_NEURON_VARS] = L->nvars.size() * 4;
    by[SZSNN_L_INPUT_PARAMS] = L->iparams.size() * 4;
    by[SZSNN_L_INPUT_VARS] = L->ivars.size() * 4;
    by[SZSNN_L_TARGETS] = L->targets.size() * 4;
    by[SZSNN_L_WEIGHTS] = L->weights.size() * 4;
    by[SZSNN_L_DELAY_BITS] = L->delay_bits.size() * 8;
    by[SZSNN_L_GROUP_PTRS] = L->group_ptrs.size() * 4;
    by[SZSNN_L_GROUP_MATRIX] = L->group_matrix.size() * 4;
    by[SZSNN_L_GQ_COUNTER] = align_up(Pt * 2, 32) * 4;
    by[SZSNN_L_GQ_BUNDLES] = Pt * 2 * max_incoming * 4;
    by[SZSNN_L_LQ_COUNTER] = Pt * D * 4;
    by[SZSNN_L_LQ_ENTRIES] = Pt * D * lq_width * 4;
    by[SZSNN_L_FIRED] = Pt * MPS * 4;
    by[SZSNN_L_FIRED_COUNT] = Pt * 4;
    by[SZSNN_L_FIRED_INPUT] = Pt * bvwp * 4;
    by[SZSNN_L_FIRED_OUTPUT] = Pt * bvwp * 4;
    by[SZSNN_L_INPUT_CURRENT] = Pt * MPS * 4;
    by[SZSNN_L_CURRENT] = 2 * Pt * MPS * 4;
    *out = L;
    return SZSNN_OK;
}

extern "C" int szsnn_layout_info_get(const szsnn_layout* L, szsnn_layout_info* info)
{
    if (!L || !info) return SZSNN_ERR_ARG;
    *info = L->info;
    return SZSNN_OK;
}

extern "C" int szsnn_layout_array(const szsnn_layout* L, int which, void* dst, size_t dst_bytes)
{
    if (!L || which < 0 || which >= SZSNN_L_COUNT) return SZSNN_ERR_ARG;
    const uint64_t need = L->info.bytes[which];
    if (dst_bytes < need || (!dst && need)) return SZSNN_ERR_ARG;
    const void* src = nullptr;
    switch (which) {
    case SZSNN_L_PARTITION_SIZES: src = L->partition_sizes.data(); break;
    case SZSNN_L_NEURON_PARAMS: src = L->nparams.data(); break;
    case SZSNN_L_NEURON_VARS: src = L->nvars.data(); break;
    case SZSNN_L_INPUT_PARAMS: src = L->iparams.data(); break;
    case SZSNN_L_INPUT_VARS: src = L->ivars.data(); break;
    case SZSNN_L_TARGETS: src = L->targets.data(); break;
    case SZSNN_L_WEIGHTS: src = L->weights.data(); break;
    case SZSNN_L_DELAY_BITS: src = L->delay_bits.data(); break;
    case SZSNN_L_GROUP_PTRS: src = L->group_ptrs.data(); break;
    case SZSNN_L_GROUP_MATRIX: src = L->group_matrix.data(); break;
    default: src = nullptr; break;  // queues, spikes, currents start zeroed
    }
    if (!need) return SZSNN_OK;
    if (src) std::memcpy(dst, src, need);
    else std::memset(dst, 0, need);
    return SZSNN_OK;
}

extern "C" int szsnn_layout_free(szsnn_layout* L)
{
    delete L;
    return SZSNN_OK;
}
