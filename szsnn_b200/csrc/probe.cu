// probe.cu -- measured on-chip ceilings for the step's roofline.
//
// The step's working set besides the synapse stream (neuron state and the
// per-step input accumulators, 48 MB at 1M neurons) stays in the 126 MB L2
// across steps, and every synaptic event is one fp32 reduction into an input
// accumulator at a random target.  HBM bandwidth therefore does not bound
// either part; these two probes measure what does, on the device at hand:
//
//  * L2 copy bandwidth: a float4 grid-stride copy between two 16 MB buffers
//    (both resident in L2), repeated `passes` times inside one launch so
//    launch gaps do not count; loads bypass L1 (ld.global.cg), so every pass
//    moves its bytes between L2 and the SMs; read + write bytes per second;
//  * random reductions: `red.global.add.f32` at hashed addresses into two
//    arrays of n_targets floats (the exc / inh accumulators of an n-neuron
//    network), reductions per second.  No loads feed them, so this is the
//    L2 atomic units' throughput for that footprint.
//
// Both are timed with CUDA events on the context's stream after warm-up
// passes; nothing here reads or writes any network.
#include "common.cuh"

namespace {

__global__ void __launch_bounds__(256) k_probe_copy(const float4* __restrict__ a, float4* __restrict__ b, int64_t n4,
                                                    int passes)
{
    for (int r = 0; r < passes; ++r)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x)
            b[i] = __ldcg(&a[i]);
}

// 32-bit mix (the finaliser of MurmurHash3), for probe addresses only
__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(256) k_probe_red(float* __restrict__ acc, uint32_t n_slots, int per_thread,
                                                   uint32_t salt)
{
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < per_thread; ++k) {
        const uint32_t h = mix32(tid * 0x9E3779B9u + (uint32_t)k * 0x7F4A7C15u + salt);
        atomicAdd(&acc[h % n_slots], 1.0f);
    }
}

}  // namespace

extern "C" int szsnn_probe_peaks(szsnn_ctx* ctx, int64_t n_targets, szsnn_peaks* out)
{
    if (!ctx || !out || n_targets < 1 || n_targets > (1ll << 30))
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_probe_peaks: bad arguments");
    cudaStream_t st = ctx->stream;
    const int sms = ctx->num_sms > 0 ? ctx->num_sms : 148;
    const int64_t copy_bytes = 16ll << 20;
    const int64_t n4 = copy_bytes / 16;
    float4* a = nullptr;
    float4* b = nullptr;
    float* acc = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto fin = [&](int rc) {
        cudaFree(a);
        cudaFree(b);
        cudaFree(acc);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        return rc;
    };
#define P_TRY(x)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (x);                                                                             \
        if (e_ != cudaSuccess)                                                                            \
            return fin(szsnn_set_error(ctx, SZSNN_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_))); \
    } while (0)
    P_TRY(cudaMalloc((void**)&a, copy_bytes));
    P_TRY(cudaMalloc((void**)&b, copy_bytes));
    P_TRY(cudaMalloc((void**)&acc, (size_t)2 * n_targets * sizeof(float)));
    P_TRY(cudaMemsetAsync(a, 0, copy_bytes, st));
    P_TRY(cudaMemsetAsync(acc, 0, (size_t)2 * n_targets * sizeof(float), st));
    P_TRY(cudaEventCreate(&e0));
    P_TRY(cudaEventCreate(&e1));

    // L2-resident copy: 8 blocks of 256 threads per SM, 16 passes per launch,
    // 2 warm-up launches, 5 timed
    const int cgrid = sms * 8, passes = 16, creps = 5;
    for (int r = 0; r < 2; ++r) k_probe_copy<<<cgrid, 256, 0, st>>>(a, b, n4, passes);
    P_TRY(cudaGetLastError());
    P_TRY(cudaEventRecord(e0, st));
    for (int r = 0; r < creps; ++r) k_probe_copy<<<cgrid, 256, 0, st>>>(r & 1 ? b : a, r & 1 ? a : b, n4, passes);
    P_TRY(cudaGetLastError());
    P_TRY(cudaEventRecord(e1, st));
    P_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    P_TRY(cudaEventElapsedTime(&ms, e0, e1));
    out->l2_copy_gbs = (double)creps * passes * 2.0 * (double)copy_bytes / (ms * 1e-3) / 1e9;
    out->l2_copy_bytes = 2 * copy_bytes;

    // random reductions into 2 * n_targets floats
    const int rgrid = sms * 8, per_thread = 64, rreps = 10;
    const uint32_t slots = (uint32_t)(2 * n_targets);
    for (int r = 0; r < 2; ++r) k_probe_red<<<rgrid, 256, 0, st>>>(acc, slots, per_thread, 0x1234u + (uint32_t)r);
    P_TRY(cudaGetLastError());
    P_TRY(cudaEventRecord(e0, st));
    for (int r = 0; r < rreps; ++r)
        k_probe_red<<<rgrid, 256, 0, st>>>(acc, slots, per_thread, 0xBEEFu * (uint32_t)(r + 1));
    P_TRY(cudaGetLastError());
    P_TRY(cudaEventRecord(e1, st));
    P_TRY(cudaEventSynchronize(e1));
    P_TRY(cudaEventElapsedTime(&ms, e0, e1));
    const double reds = (double)rreps * rgrid * 256.0 * per_thread;
    out->red_per_s = reds / (ms * 1e-3);
    out->red_targets = 2 * n_targets;
#undef P_TRY
    return fin(SZSNN_OK);
}
