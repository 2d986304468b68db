// common.cuh -- shared definitions of the sm_100a SZSNN step: context, error
// handling, Philox4x32-10, and the per-neuron model rules used by both the
// drop-in reference-layout kernels and the native network kernels.
//
// Floating point: every .cu file is built with -fmad=false -ftz=true
// -prec-div=true, and each rule keeps the operand order of the reference
// kernel it restates, so fp32 results are bit-identical to an IEEE CPU run of
// the same expressions with FTZ/DAZ (the reference builds with
// -cl-denorms-are-zero -cl-single-precision-constant, Simulation.ipp:13-15,
// neuron_model_traits.hpp:42-43).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <set>
#include <vector>

#include "../../include/szsnn_cuda.h"

struct szsnn_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    szsnn_layout_consts c{};
    std::string err;
    uint32_t* d_err = nullptr;        // device sticky error: [0] code, [1] info
    bool opt_sparse_input = true;     // input kernel stores sparse spikes
    int64_t fired_output_parts = -1;  // partitions held by firedOutput (-1: all)
    bool izh_half_steps = false;
    std::set<void*> allocs;
};

int szsnn_set_error(szsnn_ctx* ctx, int code, const std::string& msg);

#define SZSNN_CUDA_TRY(ctx, call)                                                    \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            return szsnn_set_error((ctx), SZSNN_ERR_CUDA,                            \
                                   std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define SZSNN_LAUNCH_CHECK(ctx)                                                      \
    do {                                                                             \
        cudaError_t e_ = cudaGetLastError();                                         \
        if (e_ != cudaSuccess)                                                       \
            return szsnn_set_error((ctx), SZSNN_ERR_CUDA,                            \
                                   std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// record the first device-side error (code, info); later ones are dropped
__device__ __forceinline__ void dev_error(uint32_t* err, uint32_t code, uint32_t info)
{
    if (err && atomicCAS(err, 0u, code) == 0u) err[1] = info;
}

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon et al., SC'11).  Counter / key conventions:
//   Poisson draw  : ctr {index in population, step_lo, step_hi, 0x504F4953}, key = seed
//   generator     : ctr {row in block, k, stream, 0x53594E47},            key = seed
// (population- and block-relative, so a network draws the same streams
// wherever it sits in a batch)
#define SZ_PHILOX_M0 0xD2511F53u
#define SZ_PHILOX_M1 0xCD9E8D57u
#define SZ_PHILOX_W0 0x9E3779B9u
#define SZ_PHILOX_W1 0xBB67AE85u
#define SZ_STREAM_POISSON 0x504F4953u
#define SZ_STREAM_GEN 0x53594E47u

__host__ __device__ __forceinline__ uint4 sz_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                    uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(SZ_PHILOX_M0, c0), lo0 = SZ_PHILOX_M0 * c0;
        uint32_t hi1 = __umulhi(SZ_PHILOX_M1, c2), lo1 = SZ_PHILOX_M1 * c2;
#else
        uint64_t p0 = (uint64_t)SZ_PHILOX_M0 * c0, p1 = (uint64_t)SZ_PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += SZ_PHILOX_W0; k1 += SZ_PHILOX_W1;
    }
    return make_uint4(c0, c1, c2, c3);
}

__host__ __device__ __forceinline__ float sz_u24(uint32_t r) { return (float)(r >> 8) * (1.0f / 16777216.0f); }

__host__ __device__ __forceinline__ uint32_t sz_bounded(uint32_t r, uint32_t range)
{
    return (uint32_t)(((uint64_t)r * (uint64_t)range) >> 32);
}

__device__ __forceinline__ bool sz_poisson_fires(uint64_t seed, int64_t idx, int64_t step, float p)
{
    uint4 r = sz_philox((uint32_t)idx, (uint32_t)step, (uint32_t)((uint64_t)step >> 32), SZ_STREAM_POISSON,
                        (uint32_t)seed, (uint32_t)(seed >> 32));
    return sz_u24(r.x) < p;
}

// ---------------------------------------------------------------- models
// IF_curr_exp -- IF_curr_exp_update_kernel.cl:230-287.
// p: 0 v_rest 1 cm 2 tau_m 3 tau_refrac 4 tau_syn_E 5 tau_syn_I 6 i_offset 7 v_reset 8 v_thresh
// de, di: (1 - 1/tau_syn_E), (1 - 1/tau_syn_I), the same fp32 operations
// whether evaluated per step (reference layout) or once per population.
template <class P>
__device__ __forceinline__ bool sz_if_curr_exp(const P& p, float& v, float& ie, float& ii, float& fired,
                                               float in_e, float in_i, float i_ext, bool forced, float de, float di)
{
    const float one = 1.0f;
    float Ie = (de * ie) + in_e;
    float Ii = (di * ii) + in_i;
    float I = ((Ie + Ii) + i_ext) + p(6);
    ie = Ie;
    ii = Ii;
    bool refr = fired <= p(3);
    fired += one;
    float vv = v;
    if (!refr) {
        float delta = I / p(1) + (p(0) - vv) / p(2);
        vv += delta;
    }
    bool spk = ((!refr) && (vv >= p(8))) || forced;
    if (spk) { vv = p(7); fired = one; }
    v = vv;
    return spk;
}

// IF_cond_exp -- no reference kernel.  Conductances decay and integrate first
// (the order of IF_curr_exp_update_kernel.cl:230-231), inhibitory input sums
// are negative (weights split by sign as gather_kernel.cl:172) and subtract;
// then v integrates with the new conductances.  p: IF_curr_exp slots + 9 e_rev_E 10 e_rev_I
template <class P>
__device__ __forceinline__ bool sz_if_cond_exp(const P& p, float& v, float& ge, float& gi, float& fired,
                                               float in_e, float in_i, float i_ext, bool forced, float de, float di)
{
    const float one = 1.0f;
    float g_e = (de * ge) + in_e;
    float g_i = (di * gi) - in_i;
    ge = g_e;
    gi = g_i;
    bool refr = fired <= p(3);
    fired += one;
    float vv = v;
    if (!refr) {
        float I = (((g_e * (p(9) - vv)) + (g_i * (p(10) - vv))) + p(6)) + i_ext;
        float delta = I / p(1) + (p(0) - vv) / p(2);
        vv += delta;
    }
    bool spk = ((!refr) && (vv >= p(8))) || forced;
    if (spk) { vv = p(7); fired = one; }
    v = vv;
    return spk;
}

// Izhikevich -- Izhikevich_update_kernel.cl:221,259-263,275-279 (single 1 ms
// step).  half_steps: two 0.5 ms half-steps for v, then u from the new v.
template <class P>
__device__ __forceinline__ bool sz_izhikevich(const P& p, float& v, float& u, float in_e, float in_i,
                                              float i_ext, bool forced, bool half_steps)
{
    float I = (in_e + in_i) + i_ext;
    float vv = v, uu = u;
    float a = p(0), b = p(1);
    if (half_steps) {
        vv = vv + 0.5f * ((((0.04f * vv + 5.0f) * vv + 140.0f) - uu) + I);
        vv = vv + 0.5f * ((((0.04f * vv + 5.0f) * vv + 140.0f) - uu) + I);
        uu = uu + a * (b * vv - uu);
    } else {
        float dv = (((0.04f * vv + 5.0f) * vv + 140.0f) - uu) + I;
        float du = a * (b * vv - uu);
        vv += dv;
        uu += du;
    }
    bool spk = (vv >= 30.0f) || forced;
    if (spk) { vv = p(2); uu += p(3); }
    v = vv;
    u = uu;
    return spk;
}

// Const_rate -- Const_rate_update_kernel.cl:211-229
template <class P>
__device__ __forceinline__ bool sz_const_rate(const P& p, float& last, bool forced)
{
    float l = last + 1.0f;
    bool spk = (l == p(0)) || forced;
    if (spk) l = 0.0f;
    last = l;
    return spk;
}

// 1 - 1/tau in fp32 (IF_curr_exp_update_kernel.cl:230-231)
__host__ __device__ __forceinline__ float sz_decay(float tau) { return 1.0f - 1.0f / tau; }

__host__ __device__ __forceinline__ int64_t sz_div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }
