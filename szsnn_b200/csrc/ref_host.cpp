// ref_host.cpp -- a C++ host on the drop-in kernel seam, using nothing but the
// C ABI of libszsnn_cuda.so (no OpenCL, no CUDA runtime calls, no Python).
//
// It does what the reference's Simulation<float> does between its OpenCL
// calls (szsnn1.1/src/Simulation.ipp):
//   construction  layout of the network (NeuronData / SynapseData / GroupData /
//                 queues / spike buffers / currents, Simulation.ipp:108-118)
//                 built by szsnn_layout_build and uploaded (prepareGPUMemory,
//                 :130-138) with szsnn_alloc + szsnn_h2d;
//   each cycle    gather, the firing input, the update kernel, scatter, with
//                 the cycle argument = cycles done (step, :471-496), then the
//                 firedOutput bitvector read back and turned into ascending
//                 neuron ids (SpikeBuffer::getOutput / bitvectorToSparse,
//                 SpikeBuffer.cpp:136-165).
// A maintainer replacing the reference's OpenCL Context with the C ABI makes
// the same calls from Context::enqueueKernel; this program is that call
// sequence, runnable on its own.
//
//   szsnn_ref_host <network file> <output file>
//
// Network file (little-endian): "SZRH0001", then uint32 model (0 IF_curr_exp,
// 2 Izhikevich), mps, tpg, max_delay, n_neurons, param_count, var_count,
// cycles, forced_cycles; uint64 n_synapses; float params[n][pc],
// vars[n][vc]; uint32 src[s], tgt[s]; float w[s]; uint32 delay1[s]; then per
// forced cycle: uint32 cycle, count, ids[count].
// Output file: per cycle uint32 count, ids[count]; then float vars[vc][n].
#include "szsnn_cuda.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace {

struct Fail {
    std::string msg;
};

void check(int rc, szsnn_ctx* ctx, const char* what)
{
    if (rc) throw Fail{std::string(what) + ": status " + std::to_string(rc) + ": " + (ctx ? szsnn_last_error(ctx) : "")};
}

template <class T>
void rd(FILE* f, T* dst, size_t n)
{
    if (n && std::fread(dst, sizeof(T), n, f) != n) throw Fail{"network file truncated"};
}

template <class T>
T rd1(FILE* f)
{
    T v{};
    rd(f, &v, 1);
    return v;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <network file> <output file>\n", argv[0]);
        return 2;
    }
    szsnn_ctx* ctx = nullptr;
    szsnn_layout* lay = nullptr;
    std::vector<void*> dev(SZSNN_L_COUNT, nullptr);
    int status = 0;
    try {
        FILE* f = std::fopen(argv[1], "rb");
        if (!f) throw Fail{"cannot open the network file"};
        char magic[8];
        rd(f, magic, 8);
        if (std::memcmp(magic, "SZRH0001", 8) != 0) throw Fail{"not a network file"};
        const uint32_t model = rd1<uint32_t>(f), mps = rd1<uint32_t>(f), tpg = rd1<uint32_t>(f);
        const uint32_t max_delay = rd1<uint32_t>(f), n = rd1<uint32_t>(f), pc = rd1<uint32_t>(f);
        const uint32_t vc = rd1<uint32_t>(f), cycles = rd1<uint32_t>(f), forced_cycles = rd1<uint32_t>(f);
        const uint64_t ns = rd1<uint64_t>(f);
        std::vector<float> params((size_t)n * pc), vars((size_t)n * vc), w(ns);
        std::vector<uint32_t> src(ns), tgt(ns), d1(ns);
        rd(f, params.data(), params.size());
        rd(f, vars.data(), vars.size());
        rd(f, src.data(), ns);
        rd(f, tgt.data(), ns);
        rd(f, w.data(), ns);
        rd(f, d1.data(), ns);
        std::map<uint32_t, std::vector<uint32_t>> forced;
        for (uint32_t k = 0; k < forced_cycles; ++k) {
            const uint32_t c = rd1<uint32_t>(f), cnt = rd1<uint32_t>(f);
            std::vector<uint32_t> ids(cnt);
            rd(f, ids.data(), cnt);
            forced[c] = ids;
        }
        std::fclose(f);

        // Context::setup with the layout constants locales.h holds
        szsnn_layout_consts consts{mps, tpg, 32, max_delay};
        check(szsnn_ctx_create(0, &consts, &ctx), nullptr, "szsnn_ctx_create");
        // the layout Simulation's constructor builds
        szsnn_layout_desc desc{};
        desc.n_neurons = n;
        desc.neuron_param_count = pc;
        desc.neuron_var_count = vc;
        desc.neuron_params = params.data();
        desc.neuron_vars = vars.data();
        desc.n_synapses = ns;
        desc.src = src.data();
        desc.tgt = tgt.data();
        desc.weight = w.data();
        desc.delay1 = d1.data();
        desc.add_phony_synapse = 1;
        char err[512];
        int rc = szsnn_layout_build(&consts, &desc, &lay, err, sizeof(err));
        if (rc) throw Fail{std::string("szsnn_layout_build: ") + err};
        szsnn_layout_info info{};
        check(szsnn_layout_info_get(lay, &info), ctx, "szsnn_layout_info_get");
        // createBuffer + writeBuffer for every array (prepareGPUMemory)
        for (int k = 0; k < SZSNN_L_COUNT; ++k) {
            const size_t bytes = (size_t)info.bytes[k];
            std::vector<unsigned char> host(bytes ? bytes : 16, 0);
            if (bytes) check(szsnn_layout_array(lay, k, host.data(), bytes), ctx, "szsnn_layout_array");
            check(szsnn_alloc(ctx, host.size(), &dev[k]), ctx, "szsnn_alloc");
            check(szsnn_h2d(ctx, dev[k], host.data(), host.size()), ctx, "szsnn_h2d");
        }
        auto U = [&](int k) { return static_cast<uint32_t*>(dev[k]); };
        auto F = [&](int k) { return static_cast<float*>(dev[k]); };
        const uint32_t pn = info.neuron_partitions, ptot = info.total_partitions, bvwp = mps / 32;
        auto update = model == 2 ? szsnn_update_izhikevich : szsnn_update_if_curr_exp;

        FILE* out = std::fopen(argv[2], "wb");
        if (!out) throw Fail{"cannot open the output file"};
        std::vector<uint32_t> words((size_t)pn * bvwp);
        uint32_t is_input = 0;
        for (uint32_t c = 0; c < cycles; ++c) {
            // prefire: gather (Simulation.ipp:402-420)
            check(szsnn_gather(ctx, c, ptot, U(SZSNN_L_PARTITION_SIZES), F(SZSNN_L_CURRENT), info.gq_pitch,
                               U(SZSNN_L_GQ_COUNTER), U(SZSNN_L_GQ_BUNDLES), U(SZSNN_L_TARGETS), F(SZSNN_L_WEIGHTS)),
                  ctx, "szsnn_gather");
            // SpikeBuffer::setInput: a non-empty list replaces the input bitvector
            auto it = forced.find(c);
            if (it != forced.end()) {
                std::vector<uint32_t> vec((size_t)ptot * bvwp, 0);
                for (uint32_t id : it->second) vec[(id / mps) * bvwp + (id % mps) / 32] |= 1u << (id % 32);
                check(szsnn_h2d(ctx, dev[SZSNN_L_FIRED_INPUT], vec.data(), vec.size() * 4), ctx, "szsnn_h2d");
                is_input = 1;
            } else {
                is_input = 0;
            }
            // fire: the update kernel (:423-441)
            check(update(ctx, c, pn, U(SZSNN_L_PARTITION_SIZES), F(SZSNN_L_NEURON_PARAMS), F(SZSNN_L_NEURON_VARS), 0,
                         F(SZSNN_L_INPUT_CURRENT), F(SZSNN_L_CURRENT), is_input, U(SZSNN_L_FIRED_INPUT),
                         U(SZSNN_L_FIRED_COUNT), U(SZSNN_L_FIRED), U(SZSNN_L_FIRED_OUTPUT), 0, ptot),
                  ctx, "szsnn_update");
            // postfire: scatter (:444-460)
            check(szsnn_scatter(ctx, c, ptot, U(SZSNN_L_FIRED_COUNT), U(SZSNN_L_FIRED), info.group_pitch,
                                info.group_step, U(SZSNN_L_GROUP_PTRS), U(SZSNN_L_GROUP_MATRIX), info.gq_pitch,
                                U(SZSNN_L_GQ_COUNTER), U(SZSNN_L_GQ_BUNDLES), U(SZSNN_L_LQ_COUNTER),
                                static_cast<int16_t*>(dev[SZSNN_L_LQ_ENTRIES]),
                                static_cast<const uint64_t*>(dev[SZSNN_L_DELAY_BITS])),
                  ctx, "szsnn_scatter");
            // stepAndFired: firedOutput of the neuron partitions as ascending ids
            check(szsnn_d2h(ctx, words.data(), dev[SZSNN_L_FIRED_OUTPUT], words.size() * 4), ctx, "szsnn_d2h");
            std::vector<uint32_t> ids;
            for (uint32_t p = 0; p < pn; ++p)
                for (uint32_t wi = 0; wi < bvwp; ++wi)
                    for (uint32_t b = 0, x = words[(size_t)p * bvwp + wi]; x; ++b, x >>= 1)
                        if (x & 1u) ids.push_back(p * mps + wi * 32 + b);
            const uint32_t cnt = (uint32_t)ids.size();
            std::fwrite(&cnt, 4, 1, out);
            if (cnt) std::fwrite(ids.data(), 4, cnt, out);
        }
        check(szsnn_sync(ctx), ctx, "szsnn_sync");
        // neuron variables back in [var][neuron] order: layout [vc][Pn][MPS], ids p*MPS + i
        std::vector<float> v((size_t)vc * pn * mps);
        check(szsnn_d2h(ctx, v.data(), dev[SZSNN_L_NEURON_VARS], v.size() * 4), ctx, "szsnn_d2h");
        for (uint32_t k = 0; k < vc; ++k)
            std::fwrite(v.data() + (size_t)k * pn * mps, 4, n, out);  // ids 0..n-1 are p*MPS+i in order
        std::fclose(out);
    } catch (const Fail& e) {
        std::fprintf(stderr, "szsnn_ref_host: %s\n", e.msg.c_str());
        status = 1;
    }
    for (void* p : dev)
        if (p && ctx) szsnn_free(ctx, p);
    if (lay) szsnn_layout_free(lay);
    if (ctx) szsnn_ctx_destroy(ctx);
    return status;
}
