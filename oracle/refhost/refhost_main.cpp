// refhost_main.cpp -- TEST INFRASTRUCTURE: the reference's own host code
// (NetworkGraph, NeuronData, SynapseData, GroupData, the queues,
// SpikeBuffer, CurrentData, Simulation<float>; compiled unchanged where the
// reference's sources lie) driven through the szsnn compat layer
// (szsnn_b200/compat: cl.hpp, std-backed Boost, Context.cpp over the C ABI).
//
//   refhost layout <spec> <out>   build the reference layout on the host
//                                 (no device) and write its arrays
//   refhost run <spec> <out>      Simulation<float> on the sm_100a drop-in
//                                 kernels: stepAndFired(fInput) per step,
//                                 the firing output of every step and the
//                                 final neuron variables written out
//
// <spec> (little endian, written by tests/refhost.py):
//   "SZRH" u32 version=1, u32 model (0 IF_curr_exp, 1 Izhikevich),
//   u32 n_neurons, u32 n_inputs, u32 steps, u64 n_syn,
//   f32 params[n][param_count], f32 vars[n][var_count],
//   f32 input_rate[n_inputs] (Const_rate parameter),
//   u32 src[n_syn] (>= n_neurons: input src - n_neurons), u32 tgt[n_syn],
//   f32 w[n_syn], u32 delay[n_syn] (the user delay NetworkGraph takes),
//   per step: u32 k, u32 ids[k] (firing input, the reference's global ids)
// <out>: a sequence of records  u32 name_len, name, u32 elem_size, u64 count, bytes
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Simulation.hpp"
#include "NetworkGraph.hpp"
#include "models/Const_rate_InputModel.hpp"
#include "models/IF_curr_exp_NeuronModel.hpp"
#include "models/Izhikevich_NeuronModel.hpp"
#include "models/NONE_NeuronModel.hpp"

namespace {

struct Spec {
    uint32_t model = 0, n = 0, ni = 0, steps = 0;
    uint64_t n_syn = 0;
    std::vector<float> params, vars, rates, w;
    std::vector<uint32_t> src, tgt, delay;
    std::vector<std::vector<uint32_t>> forced;
};

template <class T>
void rd(std::ifstream& f, T* p, size_t n)
{
    f.read(reinterpret_cast<char*>(p), (std::streamsize)(n * sizeof(T)));
    if (!f) throw std::runtime_error("spec file truncated");
}

struct Out {
    std::ofstream f;
    explicit Out(const char* path) : f(path, std::ios::binary) {}
    template <class T>
    void put(const std::string& name, const T* p, uint64_t count)
    {
        const uint32_t nl = (uint32_t)name.size(), es = (uint32_t)sizeof(T);
        f.write(reinterpret_cast<const char*>(&nl), 4);
        f.write(name.data(), nl);
        f.write(reinterpret_cast<const char*>(&es), 4);
        f.write(reinterpret_cast<const char*>(&count), 8);
        if (count) f.write(reinterpret_cast<const char*>(p), (std::streamsize)(count * sizeof(T)));
    }
    template <class T>
    void put(const std::string& name, const std::vector<T>& v) { put(name, v.data(), v.size()); }
};

Spec read_spec(const char* path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    char magic[4];
    rd(f, magic, 4);
    if (std::string(magic, 4) != "SZRH") throw std::runtime_error("not a refhost spec");
    uint32_t version = 0;
    rd(f, &version, 1);
    if (version != 1) throw std::runtime_error("unknown spec version");
    Spec s;
    rd(f, &s.model, 1);
    rd(f, &s.n, 1);
    rd(f, &s.ni, 1);
    rd(f, &s.steps, 1);
    rd(f, &s.n_syn, 1);
    const size_t pc = s.model == 0 ? 9 : 4, vc = s.model == 0 ? 4 : 2;
    s.params.resize((size_t)s.n * pc);
    s.vars.resize((size_t)s.n * vc);
    s.rates.resize(s.ni);
    rd(f, s.params.data(), s.params.size());
    rd(f, s.vars.data(), s.vars.size());
    rd(f, s.rates.data(), s.rates.size());
    s.src.resize(s.n_syn);
    s.tgt.resize(s.n_syn);
    s.w.resize(s.n_syn);
    s.delay.resize(s.n_syn);
    rd(f, s.src.data(), s.n_syn);
    rd(f, s.tgt.data(), s.n_syn);
    rd(f, s.w.data(), s.n_syn);
    rd(f, s.delay.data(), s.n_syn);
    s.forced.resize(s.steps);
    for (uint32_t t = 0; t < s.steps; ++t) {
        uint32_t k = 0;
        rd(f, &k, 1);
        s.forced[t].resize(k);
        rd(f, s.forced[t].data(), k);
    }
    return s;
}

// the network graph as NetworkCreator::fillNetworkGraph assembles it
// (NetworkCreator.hpp:118-187): neurons, inputs, neuron synapses, input
// synapses, then the input connection
template <class NM, class IM>
void fill(const Spec& s, szsnn::NetworkGraph<NM, IM>& g)
{
    const unsigned pc = szsnn::neuron_model_traits<NM>::param_count;
    const unsigned vc = szsnn::neuron_model_traits<NM>::var_count;
    for (uint32_t i = 0; i < s.n; ++i) {
        NM m;
        for (unsigned k = 0; k < pc; ++k) m.setParam(k, s.params[(size_t)i * pc + k]);
        for (unsigned k = 0; k < vc; ++k) m.setVar(k, s.vars[(size_t)i * vc + k]);
        g.addNeuron(i, m);
    }
    for (uint32_t j = 0; j < s.ni; ++j) {
        IM m;
        m.setParam(0u, s.rates[j]);
        m.setVar(0u, 0.0f);
        g.addInput(j, m);
    }
    for (int pass = 0; pass < 2; ++pass)
        for (uint64_t e = 0; e < s.n_syn; ++e) {
            const bool from_input = s.src[e] >= s.n;
            if (from_input != (pass == 1)) continue;
            szsnn::Synapse<float> sy;
            sy.sourceNeuronIdx = from_input ? s.src[e] - s.n : s.src[e];
            sy.targetNeuronIdx = s.tgt[e];
            sy.weight = s.w[e];
            sy.delay = s.delay[e];
            sy.synapseIdx = 0;
            if (from_input) g.addInputSynapse(sy);
            else g.addSynapse(sy);
        }
    if (s.ni) g.connectInput();
}

template <class T>
std::vector<uint32_t> pairs(const std::vector<T>& v)
{
    std::vector<uint32_t> out;
    out.reserve(v.size() * 2);
    for (const T& x : v) {
        out.push_back((uint32_t)x.s[0]);
        out.push_back((uint32_t)x.s[1]);
    }
    return out;
}

template <class NM, class IM>
int layout(const Spec& s, const char* out_path)
{
    szsnn::NetworkGraph<NM, IM> g;
    fill(s, g);
    // no device: host-only buffers, and no memory bookkeeping (its limits come
    // from the device, DeviceManager.cpp:36-50)
    boost::shared_ptr<szsnn::Context> ctx(new szsnn::Context(false));
    // the order of Simulation's constructor (Simulation.ipp:106-112)
    g._addPhonySynapse();
    szsnn::NeuronData<float> nd(ctx, s.ni > 0);
    nd.initialize(g);
    szsnn::SynapseData<float> sd(ctx);
    sd.initialize(g);
    Out o(out_path);
    o.put("partition_sizes", nd.getTotalPartitionSizesRef().getDataRef());
    o.put("neuron_params", nd.getNeuronParametersRef().getDataRef());
    o.put("neuron_vars", nd.getNeuronVariablesRef().getDataRef());
    if (s.ni) {
        o.put("input_params", nd.getInputParametersRef().getDataRef());
        o.put("input_vars", nd.getInputVariablesRef().getDataRef());
    }
    o.put("targets", sd.getTargetsRef().getDataRef());
    o.put("weights", sd.getWeightsRef().getDataRef());
    o.put("delay_bits", sd.getDelaysBitmapRef().getDataRef());
    o.put("group_ptrs", pairs(sd.getGroupPtrsRef().getDataRef()));
    o.put("group_matrix", pairs(sd.getGroupMatrixRef().getDataRef()));
    const uint64_t meta[3] = {(uint64_t)sd.getPitch(), (uint64_t)sd.getStep(), (uint64_t)sd.getMaxIncomingBundles()};
    o.put("pitch_step_maxbundles", meta, 3);
    return 0;
}

template <class NM, class IM>
int run(const Spec& s, const char* out_path)
{
    szsnn::NetworkGraph<NM, IM> g;
    fill(s, g);
    szsnn::Context ctx;
    ctx.setup();
    szsnn::Simulation<float> sim(ctx, g);
    Out o(out_path);
    std::vector<uint32_t> counts, ids;
    for (uint32_t t = 0; t < s.steps; ++t) {
        const std::vector<unsigned>& fired =
            s.forced[t].empty() ? sim.stepAndFired() : sim.stepAndFired(s.forced[t]);
        counts.push_back((uint32_t)fired.size());
        ids.insert(ids.end(), fired.begin(), fired.end());
    }
    o.put("fired_counts", counts);
    o.put("fired_ids", ids);
    sim.neurons.downloadFromDevice();
    o.put("neuron_vars", sim.neurons.getNeuronVariablesRef().getDataRef());
    return 0;
}

template <class NM>
int dispatch(const Spec& s, const std::string& mode, const char* out)
{
    if (s.ni) {
        typedef szsnn::Const_rate_InputModel<float> IM;
        return mode == "layout" ? layout<NM, IM>(s, out) : run<NM, IM>(s, out);
    }
    typedef szsnn::NONE_NeuronModel<float> IM;
    return mode == "layout" ? layout<NM, IM>(s, out) : run<NM, IM>(s, out);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 4 || (std::string(argv[1]) != "layout" && std::string(argv[1]) != "run")) {
        std::fprintf(stderr, "usage: refhost layout|run <spec> <out>\n");
        return 2;
    }
    try {
        const Spec s = read_spec(argv[2]);
        if (s.model == 0) return dispatch<szsnn::IF_curr_exp_NeuronModel<float>>(s, argv[1], argv[3]);
        return dispatch<szsnn::Izhikevich_NeuronModel<float>>(s, argv[1], argv[3]);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "refhost: %s\n", e.what());
        return 1;
    }
}
