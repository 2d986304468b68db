// ref_kernels.cu -- drop-in sm_100a kernels on the reference's buffer layout.
//
// Each entry point takes the argument list its OpenCL counterpart is bound with
// in Simulation::prep*Kernel (Simulation.ipp:214-340) and produces the same
// buffer contents, with a B200-native body:
//  * update: one CTA per partition, one thread per neuron (MPS <= 1024), spikes
//    compacted with warp ballot + block prefix scan (ascending neuron order) and
//    the dense bitvector written straight from the ballot word, instead of the
//    local atomic slot claim + barrier-per-chunk bitvector build
//    (IF_curr_exp_update_kernel.cl:58-94,288);
//  * gather: one CTA per target partition, warp per bundle, native shared-memory
//    fp32 atomics instead of the CAS loop (gather_kernel.cl:19-35);
//  * scatter: one thread per spike for the delay-bitmap ring push (the reference
//    walks spikes serially with one barrier each, scatter_kernel.cl:121-181) and
//    one warp per popped ring entry for the bundle fan-out.
// Queue overflow is reported through the context's sticky device error
// instead of being dropped silently (scatter_kernel.cl:158-171).
#include "common.cuh"

namespace {

struct RefUpdateArgs {
    uint64_t cycle;
    uint32_t localPartitionCount;
    const uint32_t* partitionSizes;
    const float* params;
    float* vars;
    uint32_t isInputCurrent;
    const float* inputCurrent;
    const float* current;
    uint32_t isInputFiring;
    const uint32_t* inputFired;
    uint32_t* firedCount;
    uint32_t* fired;
    uint32_t* firedOutput;
    uint32_t partitionOffset;
    uint32_t globalPartitionCount;
    uint32_t mps;
    uint32_t store_sparse;
    int64_t fired_output_parts;
    uint32_t izh_half;
    uint32_t* err;
};

// per-neuron parameter accessor on the reference SoA layout:
// params[(k * localPartitionCount + partition) * MPS + n]  (NeuronData.ipp:19-22)
struct SoaParams {
    const float* base;
    size_t step;
    __device__ __forceinline__ float operator()(int k) const { return base[(size_t)k * step]; }
};

enum { M_IF_CURR = 0, M_IZH = 2, M_CONST = 4 };

template <int MODEL>
__global__ void __launch_bounds__(1024) k_ref_update(RefUpdateArgs a)
{
    __shared__ uint32_t s_warp_cnt[32];
    __shared__ uint32_t s_warp_off[33];
    const uint32_t P = blockIdx.x;                    // CURRENT_PARTITION
    const uint32_t gP = P + a.partitionOffset;        // l_partitionIdx
    const uint32_t psize = a.partitionSizes[gP];
    const uint32_t n = threadIdx.x;
    const uint32_t lane = n & 31, warp = n >> 5;
    const uint32_t bvwp = a.mps / 32;
    const size_t step = (size_t)a.localPartitionCount * a.mps;

    bool spk = false;
    if (n < psize && n < a.mps) {
        const float* cur_e = a.current + ((size_t)0 * a.globalPartitionCount + gP) * a.mps;
        const float* cur_i = a.current + ((size_t)1 * a.globalPartitionCount + gP) * a.mps;
        float i_ext = (a.isInputCurrent == 1) ? a.inputCurrent[(size_t)gP * a.mps + n] : 0.0f;
        bool forced = (a.isInputFiring == 1) ? ((a.inputFired[(size_t)gP * bvwp + n / 32] >> (n % 32)) & 1u) : false;
        SoaParams p{a.params + (size_t)P * a.mps + n, step};
        float* var = a.vars + (size_t)P * a.mps + n;
        if (MODEL == M_IF_CURR) {
            float v = var[0], ie = var[step], ii = var[2 * step], fired = var[3 * step];
            spk = sz_if_curr_exp(p, v, ie, ii, fired, cur_e[n], cur_i[n], i_ext, forced, sz_decay(p(4)), sz_decay(p(5)));
            var[0] = v; var[step] = ie; var[2 * step] = ii; var[3 * step] = fired;
        } else if (MODEL == M_IZH) {
            float v = var[0], u = var[step];
            spk = sz_izhikevich(p, v, u, cur_e[n], cur_i[n], i_ext, forced, a.izh_half != 0);
            var[0] = v; var[step] = u;
        } else {
            float last = var[0];
            spk = sz_const_rate(p, last, forced);
            var[0] = last;
        }
    }
    const uint32_t ball = __ballot_sync(0xffffffffu, spk);
    // storeDenseSpikes: word w of the partition = neurons 32w..32w+31
    if (lane == 0 && warp < bvwp && (a.fired_output_parts < 0 || (int64_t)gP < a.fired_output_parts))
        a.firedOutput[(size_t)gP * bvwp + warp] = ball;
    if (!a.store_sparse) return;
    // storeSparseSpikes: ascending neuron order via ballot + block scan
    if (lane == 0) s_warp_cnt[warp] = __popc(ball);
    __syncthreads();
    const uint32_t nwarps = blockDim.x >> 5;
    if (warp == 0) {
        uint32_t c = lane < nwarps ? s_warp_cnt[lane] : 0u;
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        s_warp_off[lane] = incl - c;
        if (lane == 31) s_warp_off[32] = incl;
    }
    __syncthreads();
    if (spk) {
        uint32_t rank = __popc(ball & ((1u << lane) - 1u));
        a.fired[(size_t)gP * a.mps + s_warp_off[warp] + rank] = n;
    }
    if (n == 0) a.firedCount[gP] = s_warp_off[32];
}

struct RefGatherArgs {
    uint64_t cycle;
    uint32_t partitionCount;
    const uint32_t* partitionSizes;
    float* current;
    uint64_t gqPitch;
    uint32_t* gqCounter;
    const uint32_t* gqBundles;
    const uint32_t* targets;
    const float* weights;
    uint32_t mps, bundle, tpg;
    uint32_t* err;
};

__global__ void __launch_bounds__(1024) k_ref_gather(RefGatherArgs a)
{
    __shared__ float s_exc[1024];
    __shared__ float s_inh[1024];
    __shared__ uint32_t s_count;
    const uint32_t P = blockIdx.x;
    const uint32_t rslot = (uint32_t)((a.cycle & 1u) ^ 1u);  // getDBreadSlot (gather_kernel.cl:55-58)
    if (threadIdx.x == 0) {
        const size_t addr = (size_t)P * 2 + rslot;
        uint32_t c = a.gqCounter[addr];
        a.gqCounter[addr] = 0;
        if (c > a.gqPitch) { dev_error(a.err, SZSNN_DEV_QUEUE_OVERFLOW, P); c = (uint32_t)a.gqPitch; }
        s_count = c;
    }
    for (uint32_t i = threadIdx.x; i < a.mps; i += blockDim.x) { s_exc[i] = 0.0f; s_inh[i] = 0.0f; }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t* q = a.gqBundles + ((size_t)P * 2 + rslot) * a.gqPitch;
    const uint32_t cnt = s_count;
    for (uint32_t i = warp; i < cnt; i += nwarps) {
        const uint32_t b = q[i];
        if (lane < a.bundle) {
            const size_t off = (size_t)b * a.bundle + lane;
            const float w = a.weights[off];
            if (w != 0.0f) {
                const uint32_t t = a.targets[off];
                if (t < a.mps) atomicAdd(w >= 0.0f ? &s_exc[t] : &s_inh[t], w);
                else dev_error(a.err, SZSNN_DEV_BAD_TARGET, t);
            }
        }
    }
    __syncthreads();
    // gather_kernel.cl:194-199 writes the first ceil(size / TPG) * TPG entries
    const uint32_t psize = a.partitionSizes[P];
    uint32_t lim = (uint32_t)(sz_div_up(psize, a.tpg) * a.tpg);
    if (lim > a.mps) lim = a.mps;
    float* ge = a.current + ((size_t)0 * a.partitionCount + P) * a.mps;
    float* gi = a.current + ((size_t)1 * a.partitionCount + P) * a.mps;
    for (uint32_t i = threadIdx.x; i < lim; i += blockDim.x) { ge[i] = s_exc[i]; gi[i] = s_inh[i]; }
}

struct RefScatterArgs {
    uint64_t cycle;
    uint32_t partitionCount;
    const uint32_t* firedCount;
    const uint32_t* fired;
    const uint2* groupPtrs;
    const uint2* groupMatrix;
    uint64_t gqPitch;
    uint32_t* gqCounter;
    uint32_t* gqBundles;
    uint32_t* lqCounter;
    short2* lqEntries;
    const unsigned long long* delayBits;
    uint32_t mps, D;
    uint32_t* err;
};

__global__ void __launch_bounds__(1024) k_ref_scatter(RefScatterArgs a)
{
    __shared__ uint32_t s_lq[64];
    const uint32_t P = blockIdx.x;
    const uint32_t D = a.D;
    const size_t width = (size_t)sz_div_up((int64_t)a.mps * D, 32) * 32;  // LocalQueue.cpp:44
    uint32_t nf = a.firedCount[P];
    if (nf > a.mps) { if (threadIdx.x == 0) dev_error(a.err, SZSNN_DEV_QUEUE_OVERFLOW, P); nf = a.mps; }
    if (threadIdx.x < D) s_lq[threadIdx.x] = a.lqCounter[(size_t)P * D + threadIdx.x];
    __syncthreads();
    // local scatter: spike emitted at `cycle` with delay bit d lands in slot (cycle + d) % D
    for (uint32_t i = threadIdx.x; i < nf; i += blockDim.x) {
        const uint32_t neuron = a.fired[(size_t)P * a.mps + i];
        if (neuron >= a.mps) { dev_error(a.err, SZSNN_DEV_BAD_TARGET, neuron); continue; }
        unsigned long long bits = a.delayBits[(size_t)P * a.mps + neuron];
        while (bits) {
            const uint32_t d = (uint32_t)(__ffsll((long long)bits) - 1);
            bits &= bits - 1ull;
            if (d >= D) { dev_error(a.err, SZSNN_DEV_BAD_DELAY, d); continue; }
            const uint32_t slot = (uint32_t)((a.cycle + d) % D);
            const uint32_t idx = atomicAdd(&s_lq[slot], 1u);
            if (idx < width) a.lqEntries[((size_t)P * D + slot) * width + idx] = make_short2((short)neuron, (short)d);
            else dev_error(a.err, SZSNN_DEV_QUEUE_OVERFLOW, P);
        }
    }
    __syncthreads();
    const uint32_t pslot = (uint32_t)(a.cycle % D);
    uint32_t cnt = s_lq[pslot];
    if (cnt > width) cnt = (uint32_t)width;
    __syncthreads();
    if (threadIdx.x < D) a.lqCounter[(size_t)P * D + threadIdx.x] = (threadIdx.x == pslot) ? 0u : s_lq[threadIdx.x];
    // global scatter: fan each due (neuron, delay) entry out to the target
    // partitions' global queues, write slot cycle & 1 (scatter_kernel.cl:325-345)
    const uint32_t wslot = (uint32_t)(a.cycle & 1u);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const short2* ent = a.lqEntries + ((size_t)P * D + pslot) * width;
    for (uint32_t e = warp; e < cnt; e += nwarps) {
        const short2 en = ent[e];
        const uint32_t neuron = (uint32_t)(uint16_t)en.x, d = (uint32_t)(uint16_t)en.y;
        if (neuron >= a.mps || d >= D) { if (lane == 0) dev_error(a.err, SZSNN_DEV_BAD_TARGET, neuron); continue; }
        const uint2 ad = a.groupPtrs[((size_t)P * a.mps + neuron) * D + d];
        for (uint32_t k = lane; k < ad.y; k += 32) {
            const uint2 so = a.groupMatrix[(size_t)ad.x + k];
            if (so.x >= a.partitionCount) { dev_error(a.err, SZSNN_DEV_BAD_TARGET, so.x); continue; }
            const uint32_t pos = atomicAdd(&a.gqCounter[(size_t)so.x * 2 + wslot], 1u);
            if (pos < a.gqPitch) a.gqBundles[((size_t)so.x * 2 + wslot) * a.gqPitch + pos] = so.y;
            else dev_error(a.err, SZSNN_DEV_QUEUE_OVERFLOW, so.x);
        }
    }
}

template <int MODEL>
int launch_ref_update(szsnn_ctx* ctx, uint64_t cycle, uint32_t lpc, const uint32_t* ps, const float* params,
                      float* vars, uint32_t iic, float* ic, float* cur, uint32_t iif, uint32_t* ifd, uint32_t* fc,
                      uint32_t* fd, uint32_t* fo, uint32_t poff, uint32_t gpc, bool sparse)
{
    if (!ctx) return SZSNN_ERR_ARG;
    if (lpc == 0) return SZSNN_OK;
    if (!ps || !params || !vars || !cur || !fo || (iic == 1 && !ic) || (iif == 1 && !ifd) || (sparse && (!fc || !fd)))
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "update kernel: null buffer argument");
    if (poff + lpc > gpc) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "update kernel: partitions exceed globalPartitionCount");
    RefUpdateArgs a{cycle, lpc, ps, params, vars, iic, ic, cur, iif, ifd, fc, fd, fo, poff, gpc,
                    ctx->c.max_partition_size, sparse ? 1u : 0u, ctx->fired_output_parts,
                    ctx->izh_half_steps ? 1u : 0u, ctx->d_err};
    k_ref_update<MODEL><<<lpc, ctx->c.max_partition_size, 0, ctx->stream>>>(a);
    SZSNN_LAUNCH_CHECK(ctx);
    return SZSNN_OK;
}

}  // namespace

extern "C" int szsnn_update_if_curr_exp(szsnn_ctx* ctx, uint64_t cycle, uint32_t lpc, const uint32_t* ps,
                                        const float* params, float* vars, uint32_t iic, float* ic, float* cur,
                                        uint32_t iif, uint32_t* ifd, uint32_t* fc, uint32_t* fd, uint32_t* fo,
                                        uint32_t poff, uint32_t gpc)
{
    return launch_ref_update<M_IF_CURR>(ctx, cycle, lpc, ps, params, vars, iic, ic, cur, iif, ifd, fc, fd, fo, poff,
                                        gpc, true);
}

extern "C" int szsnn_update_izhikevich(szsnn_ctx* ctx, uint64_t cycle, uint32_t lpc, const uint32_t* ps,
                                       const float* params, float* vars, uint32_t iic, float* ic, float* cur,
                                       uint32_t iif, uint32_t* ifd, uint32_t* fc, uint32_t* fd, uint32_t* fo,
                                       uint32_t poff, uint32_t gpc)
{
    return launch_ref_update<M_IZH>(ctx, cycle, lpc, ps, params, vars, iic, ic, cur, iif, ifd, fc, fd, fo, poff,
                                    gpc, true);
}

extern "C" int szsnn_update_const_rate(szsnn_ctx* ctx, uint64_t cycle, uint32_t lpc, const uint32_t* ps,
                                       const float* params, float* vars, uint32_t iic, float* ic, float* cur,
                                       uint32_t iif, uint32_t* ifd, uint32_t* fc, uint32_t* fd, uint32_t* fo,
                                       uint32_t poff, uint32_t gpc)
{
    return launch_ref_update<M_CONST>(ctx, cycle, lpc, ps, params, vars, iic, ic, cur, iif, ifd, fc, fd, fo, poff,
                                      gpc, ctx ? ctx->opt_sparse_input : false);
}

extern "C" int szsnn_gather(szsnn_ctx* ctx, uint64_t cycle, uint32_t pc, const uint32_t* ps, float* cur,
                            uint64_t gqPitch, uint32_t* gqc, uint32_t* gqb, const uint32_t* targets,
                            const float* weights)
{
    if (!ctx) return SZSNN_ERR_ARG;
    if (pc == 0) return SZSNN_OK;
    if (!ps || !cur || !gqc || (!gqb && gqPitch) || !targets || !weights)
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_gather: null buffer argument");
    RefGatherArgs a{cycle, pc, ps, cur, gqPitch, gqc, gqb, targets, weights,
                    ctx->c.max_partition_size, ctx->c.warp_size, ctx->c.threads_per_group, ctx->d_err};
    k_ref_gather<<<pc, 1024, 0, ctx->stream>>>(a);
    SZSNN_LAUNCH_CHECK(ctx);
    return SZSNN_OK;
}

extern "C" int szsnn_scatter(szsnn_ctx* ctx, uint64_t cycle, uint32_t pc, uint32_t* fc, uint32_t* fd,
                             uint32_t groupPitch, uint32_t groupStep, const uint32_t* groupPtrs,
                             const uint32_t* groupMatrix, uint64_t gqPitch, uint32_t* gqc, uint32_t* gqb,
                             uint32_t* lqc, int16_t* lqe, const uint64_t* delayBits)
{
    (void)groupPitch;
    (void)groupStep;  // the warp-per-entry fan-out needs no pitch/step packing
    if (!ctx) return SZSNN_ERR_ARG;
    if (pc == 0) return SZSNN_OK;
    if (!fc || !fd || !groupPtrs || !groupMatrix || !gqc || (!gqb && gqPitch) || !lqc || !lqe || !delayBits)
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_scatter: null buffer argument");
    RefScatterArgs a{cycle, pc, fc, fd, (const uint2*)groupPtrs, (const uint2*)groupMatrix, gqPitch, gqc, gqb,
                     lqc, (short2*)lqe, (const unsigned long long*)delayBits,
                     ctx->c.max_partition_size, ctx->c.max_synaptic_delay, ctx->d_err};
    k_ref_scatter<<<pc, 512, 0, ctx->stream>>>(a);
    SZSNN_LAUNCH_CHECK(ctx);
    return SZSNN_OK;
}
