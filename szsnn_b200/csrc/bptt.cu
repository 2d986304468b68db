// bptt.cu -- differentiable IF_curr_exp RNN: forward with checkpoints and the
// hand-written BPTT adjoint.  No reference counterpart (the reference has no
// training path); the forward rule is IF_curr_exp_update_kernel.cl:230-287
// with dt folded to 1 and tau_refrac 0, the exc / inh channel of a weight is
// its sign (gather_kernel.cl:172-178).  Per trial b, neuron i, step t:
//   a_t = sum_j x_t[j] Win+[j,i] + sum_j s_{t-1}[j] Wrec+[j,i]   (c_t: negative parts)
//   Ie_t = de Ie_{t-1} + a_t ;  Ii_t = di Ii_{t-1} + c_t
//   u_t  = v_{t-1} + ((Ie_t + Ii_t) + i_offset)/cm + (v_rest - v_{t-1})/tau_m
//   s_t  = u_t >= v_thresh ;  v_t = s_t ? v_reset : u_t
//   y_t  = alpha y_{t-1} + sum_i s_t[i] Wout[i,k] ;  ymax = max_t y_t ;  vsum = sum_t v_t
// The gradient is exact except dH/du, replaced by the fast sigmoid surrogate
// 1/(1 + beta|u - v_thresh|)^2 (SuperSpike, Zenke & Ganguli 2018); beta <= 0
// gives dH/du = 0.  Forward spikes are kept; the backward recomputes u_t
// segment by segment from checkpoints taken every `checkpoint_every` steps.
//
// Kernels (all fp32, deterministic summation order, no atomics except the
// small readout-weight gradient):
//   k_bptt_step     one launch per step: per-trial active input / spike lists
//                   compacted in shared memory (ascending), dense gather of
//                   their weight rows (4 neurons per thread, float4 rows, 8
//                   loads in flight, added in list order), the neuron update,
//                   spike bitmap, and the readout + running max of step t-1
//   k_bptt_spmm     R[j,b] = sum_k w_jk lam_{sign(w)}[k,b] over the CSR rows of
//                   Wrec: the sign is folded into the column index of the
//                   stacked [lam_e; lam_i] rows, half a warp per synapse, four
//                   trials per lane (float4); the same lambda rows give the
//                   recurrent weight gradient of that step (masked trial sum)
//   k_bptt_adjoint  reverse-time update of (lam_u, lam_Ie, lam_Ii) per (b,i)
//   k_bptt_dwin     input weight gradient, one owner per weight
#include "common.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

constexpr int BP_BLOCK = 256;

struct BpttK {
    int B, N, M, K, T, ck, Nw, Mw;
    float v_rest, cm, tau_m, i_offset, v_reset, v_thresh, alpha, beta, de, di, km;
    const float* w_in;
    const float* w_rec;       // dense [N][N] built from the CSR
    const long long* rp;      // CSR rows of Wrec (presynaptic)
    const int* col;
    const float* val;
    const float* w_out;
    const uint32_t* x_bits;   // [T][B][Mw]
    uint32_t* spikes;         // [T][B][Nw]
    float* Ie;
    float* Ii;
    float* v;
    float* y;                 // [B][K]
    float* ymax;
    int* tmax;
    float* vsum;
    float* u_seg;             // [ck][B][N]
    float* u_trace;           // [T][B][N] pre-reset membrane of the forward, or null
};

// ascending list of the set bits of words[0..nwords) (bits < nbits) into out;
// returns the count (all threads).  s_tmp: >= 33 ints of shared memory.
__device__ int block_compact(const uint32_t* words, int nwords, int nbits, int* out, int* s_tmp)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    int base = 0;
    for (int c0 = 0; c0 < nwords; c0 += blockDim.x) {
        const int w = c0 + tid;
        const uint32_t word = (w < nwords) ? words[w] : 0u;
        const int cnt = __popc(word);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_tmp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int x = lane < nw ? s_tmp[lane] : 0;
            int inc2 = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, inc2, o);
                if (lane >= o) inc2 += y;
            }
            if (lane < nw) s_tmp[lane] = inc2 - x;
            if (lane == 31) s_tmp[32] = inc2;
        }
        __syncthreads();
        int pos = base + s_tmp[warp] + incl - cnt;
        uint32_t bits = word;
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1u;
            const int id = w * 32 + b;
            if (id < nbits) out[pos] = id;
            ++pos;
        }
        base += s_tmp[32];
        __syncthreads();
    }
    return base;
}

constexpr int BP_NPT = 4;  // neurons per thread in the step kernel

__device__ __forceinline__ void split_add(float w, float& e, float& c)
{
    if (w != 0.0f) { if (w >= 0.0f) e += w; else c += w; }
}

// gather the weight rows listed in `ids` (n of them) at columns i0..i0+3,
// summing positive and negative weights separately in list order
__device__ __forceinline__ void gather_rows(const float* __restrict__ W, size_t stride, const int* ids, int n, int i0,
                                            float4& e, float4& c)
{
    for (int q0 = 0; q0 < n; q0 += 8) {
        float4 wv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            wv[u] = (q0 + u < n) ? __ldg(reinterpret_cast<const float4*>(W + (size_t)ids[q0 + u] * stride + i0))
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            split_add(wv[u].x, e.x, c.x);
            split_add(wv[u].y, e.y, c.y);
            split_add(wv[u].z, e.z, c.z);
            split_add(wv[u].w, e.w, c.w);
        }
    }
}

__device__ __forceinline__ bool neuron_step(const BpttK& k, float e, float c, float& ie, float& ii, float& v, float& u)
{
    ie = (k.de * ie) + e;
    ii = (k.di * ii) + c;
    const float I = (ie + ii) + k.i_offset;
    const float v0 = v;
    u = v0 + (I / k.cm + (k.v_rest - v0) / k.tau_m);
    const bool spk = u >= k.v_thresh;
    v = spk ? k.v_reset : u;
    return spk;
}

// one forward step t (update when t < T), readout of step t-1 (block x == 0);
// recompute mode: no spike / readout / vsum writes, u stored at u_seg[t - t0]
__global__ void __launch_bounds__(BP_BLOCK) k_bptt_step(BpttK k, int t, int recompute, int t0)
{
    extern __shared__ int s_list[];
    __shared__ int s_tmp[40];
    const int b = blockIdx.y;
    int* s_x = s_list;
    int* s_s = s_list + k.M;
    int nx = 0, ns = 0;
    if (t < k.T) nx = block_compact(k.x_bits + ((size_t)t * k.B + b) * k.Mw, k.Mw, k.M, s_x, s_tmp);
    if (t >= 1) ns = block_compact(k.spikes + ((size_t)(t - 1) * k.B + b) * k.Nw, k.Nw, k.N, s_s, s_tmp);
    // readout of step t-1 (forward only): y = alpha y + sum_{j spiking} Wout[j, :]
    if (!recompute && t >= 1 && blockIdx.x == 0 && threadIdx.x < k.K) {
        const int kk = threadIdx.x;
        float acc = 0.0f;
        for (int q = 0; q < ns; ++q) acc += k.w_out[(size_t)s_s[q] * k.K + kk];
        const float yv = k.alpha * k.y[b * k.K + kk] + acc;
        k.y[b * k.K + kk] = yv;
        if (t - 1 == 0 || yv > k.ymax[b * k.K + kk]) { k.ymax[b * k.K + kk] = yv; k.tmax[b * k.K + kk] = t - 1; }
    }
    if (t >= k.T) return;
    const int lane = threadIdx.x & 31;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * BP_NPT;
    uint32_t nib = 0;
    if (i0 < k.N) {
        float4 e = make_float4(0.f, 0.f, 0.f, 0.f), c = e;
        gather_rows(k.w_in, (size_t)k.N, s_x, nx, i0, e, c);
        gather_rows(k.w_rec, (size_t)k.N, s_s, ns, i0, e, c);
        const size_t o = (size_t)b * k.N + i0;
        float4 ie = *reinterpret_cast<const float4*>(k.Ie + o);
        float4 ii = *reinterpret_cast<const float4*>(k.Ii + o);
        float4 v = *reinterpret_cast<const float4*>(k.v + o);
        float4 u;
        nib |= neuron_step(k, e.x, c.x, ie.x, ii.x, v.x, u.x) ? 1u : 0u;
        nib |= neuron_step(k, e.y, c.y, ie.y, ii.y, v.y, u.y) ? 2u : 0u;
        nib |= neuron_step(k, e.z, c.z, ie.z, ii.z, v.z, u.z) ? 4u : 0u;
        nib |= neuron_step(k, e.w, c.w, ie.w, ii.w, v.w, u.w) ? 8u : 0u;
        *reinterpret_cast<float4*>(k.Ie + o) = ie;
        *reinterpret_cast<float4*>(k.Ii + o) = ii;
        *reinterpret_cast<float4*>(k.v + o) = v;
        if (recompute) {
            *reinterpret_cast<float4*>(k.u_seg + ((size_t)(t - t0) * k.B + b) * k.N + i0) = u;
        } else {
            float4 vs = *reinterpret_cast<const float4*>(k.vsum + o);
            vs.x += v.x; vs.y += v.y; vs.z += v.z; vs.w += v.w;
            *reinterpret_cast<float4*>(k.vsum + o) = vs;
            if (k.u_trace) *reinterpret_cast<float4*>(k.u_trace + ((size_t)t * k.B + b) * k.N + i0) = u;
        }
    }
    if (!recompute) {
        // lane L holds neurons 4L..4L+3 of the warp's 128: bits 4(L%8).. of word L/8
        uint32_t word = nib << (4 * (lane & 7));
        word |= __shfl_xor_sync(0xffffffffu, word, 1);
        word |= __shfl_xor_sync(0xffffffffu, word, 2);
        word |= __shfl_xor_sync(0xffffffffu, word, 4);
        const int wd = (blockIdx.x * blockDim.x * BP_NPT + (threadIdx.x >> 5) * 32 * BP_NPT) / 32 + (lane >> 3);
        if ((lane & 7) == 0 && wd < k.Nw) k.spikes[((size_t)t * k.B + b) * k.Nw + wd] = word;
    }
}

struct BpttBwd {
    float* lam_u;      // [B][N] lam_u of step t+1, then of step t
    float* lam_e;      // [B][N] total dL/dIe of step t+1, then of step t
    float* lam_i;
    float* lamS;       // [2N][Bp] this step's (lam_e; lam_i), trial-minor
    float* lamT;       // [2][B][N] the same, neuron-minor (this step's parity half of a [2][2][B][N] buffer)
    const float* R;    // [N][Bp] recurrent term from step t+1
    float* lam_y;      // [B][K] of this step
    const float* lam_y_next;  // [B][K] of step t+1
    const int* col_sel;       // [nnz] column + N for negative weights
    const float* g_ymax;
    const float* g_vsum;
    float* dw_in;      // [M][N]
    float* dw_rec;     // [nnz]
    float* dw_out;     // [N][K]
    int Bp;
};

__device__ __forceinline__ float surrogate(float x, float beta)
{
    if (beta <= 0.0f) return 0.0f;
    const float d = 1.0f + beta * fabsf(x);
    return 1.0f / (d * d);
}

__global__ void k_bptt_colsel(const int* col, const float* val, long long nnz, int N, int* col_sel)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (long long)gridDim.x * blockDim.x)
        col_sel[q] = col[q] + (val[q] < 0.0f ? N : 0);
}

// trials (bit b) in which input / neuron j spiked, from words [B][W] of one step
__device__ __forceinline__ unsigned long long trial_mask(const uint32_t* words, int B, int W, int j, int lane)
{
    const bool on0 = lane < B && ((words[(size_t)lane * W + (j >> 5)] >> (j & 31)) & 1u);
    const bool on1 = lane + 32 < B && ((words[(size_t)(lane + 32) * W + (j >> 5)] >> (j & 31)) & 1u);
    const uint32_t b0 = __ballot_sync(0xffffffffu, on0), b1 = __ballot_sync(0xffffffffu, on1);
    return (unsigned long long)b0 | ((unsigned long long)b1 << 32);
}

// One warp per row j of Wrec, half a warp per synapse, four trials per lane:
//   R[j][b] = sum over the row of w * lamS_next[col_sel][b]
// and, with dw: the recurrent weight gradient of the step whose lambdas these
// are, dWrec[e] += sum over trials b with s_step[b][j] of lamS_next[col_sel[e]][b]
// (the same lambda row serves both; the trial sum is a fixed-order reduction
// over the half warp).
__global__ void __launch_bounds__(BP_BLOCK) k_bptt_spmm(BpttK k, const int* __restrict__ col_sel, int Bp,
                                                        const float* __restrict__ lamS, float* __restrict__ R,
                                                        float* __restrict__ dw, int s_step)
{
    __shared__ float s_dw[BP_BLOCK];
    const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15, warp = threadIdx.x >> 5;
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (j >= k.N) return;
    const unsigned long long mask =
        dw ? trial_mask(k.spikes + (size_t)s_step * k.B * k.Nw, k.B, k.Nw, j, lane) : 0ull;
    const uint32_t mb = (uint32_t)(mask >> (4 * hl)) & 0xFu;  // this lane's four trials
    const long long a = k.rp[j], e = k.rp[j + 1];
    const bool act = 4 * hl < Bp;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (long long k0 = a; k0 < e; k0 += 32) {
        const long long kk = k0 + lane;
        const float w = kk < e ? __ldg(&k.val[kk]) : 0.0f;
        const int cs = kk < e ? __ldg(&col_sel[kk]) : 0;
        const float dw_old = (mask && kk < e && w != 0.0f) ? dw[kk] : 0.0f;
#pragma unroll  // all 16 synapse pairs of the chunk: their lambda loads in flight together
        for (int q = 0; q < 32; q += 2) {
            const float wq = __shfl_sync(0xffffffffu, w, q + half);
            const int cq = __shfl_sync(0xffffffffu, cs, q + half);
            float part = 0.0f;
            if (act && wq != 0.0f) {
                const float4 l = __ldg(reinterpret_cast<const float4*>(lamS + (size_t)cq * Bp) + hl);
                acc.x += wq * l.x;
                acc.y += wq * l.y;
                acc.z += wq * l.z;
                acc.w += wq * l.w;
                part = (((mb & 1u) ? l.x : 0.0f) + ((mb & 2u) ? l.y : 0.0f)) +
                       (((mb & 4u) ? l.z : 0.0f) + ((mb & 8u) ? l.w : 0.0f));
            }
            if (mask) {  // warp-uniform
                part += __shfl_xor_sync(0xffffffffu, part, 8);
                part += __shfl_xor_sync(0xffffffffu, part, 4);
                part += __shfl_xor_sync(0xffffffffu, part, 2);
                part += __shfl_xor_sync(0xffffffffu, part, 1);
                if (hl == 0) s_dw[warp * 32 + q + half] = part;
            }
        }
        if (mask) {
            __syncwarp();
            if (kk < e && w != 0.0f) dw[kk] = dw_old + s_dw[warp * 32 + lane];
            __syncwarp();
        }
    }
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, 16);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, 16);
    acc.z += __shfl_down_sync(0xffffffffu, acc.z, 16);
    acc.w += __shfl_down_sync(0xffffffffu, acc.w, 16);
    if (R && half == 0 && act) reinterpret_cast<float4*>(R + (size_t)j * Bp)[hl] = acc;
}

__global__ void __launch_bounds__(BP_BLOCK) k_bptt_adjoint(BpttK k, BpttBwd g, int t, int t0, int have_R)
{
    __shared__ float s_ly[64];
    const int b = blockIdx.y;
    if (threadIdx.x < k.K) {
        const int kk = threadIdx.x;
        float ly = k.alpha * g.lam_y_next[b * k.K + kk];
        if (k.tmax[b * k.K + kk] == t) ly += g.g_ymax ? g.g_ymax[b * k.K + kk] : 0.0f;
        s_ly[kk] = ly;
        if (blockIdx.x == 0) g.lam_y[b * k.K + kk] = ly;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k.N) return;
    const size_t o = (size_t)b * k.N + i;
    const float u = k.u_seg[((size_t)(t - t0) * k.B + b) * k.N + i];
    const bool s = (k.spikes[((size_t)t * k.B + b) * k.Nw + (i >> 5)] >> (i & 31)) & 1u;
    float ro = 0.0f;
    for (int kk = 0; kk < k.K; ++kk) ro += k.w_out[(size_t)i * k.K + kk] * s_ly[kk];
    const float Gv = (g.g_vsum ? g.g_vsum[o] : 0.0f) + k.km * g.lam_u[o];
    const float rec = have_R ? g.R[(size_t)i * g.Bp + b] : 0.0f;
    const float Gs = ro + rec + Gv * (k.v_reset - u);
    const float lu = Gv * (s ? 0.0f : 1.0f) + Gs * surrogate(u - k.v_thresh, k.beta);
    const float le = lu / k.cm + k.de * g.lam_e[o];
    const float li = lu / k.cm + k.di * g.lam_i[o];
    g.lam_u[o] = lu;
    g.lam_e[o] = le;
    g.lam_i[o] = li;
    g.lamS[(size_t)i * g.Bp + b] = le;
    g.lamS[((size_t)k.N + i) * g.Bp + b] = li;
    g.lamT[o] = le;
    g.lamT[(size_t)k.B * k.N + o] = li;
    if (s)
        for (int kk = 0; kk < k.K; ++kk) atomicAdd(&g.dw_out[(size_t)i * k.K + kk], s_ly[kk]);
}


constexpr int DWIN_J = 16;  // inputs per dwin block

// dWin[j][i] += sum over trials with x_t[b][j] of lam_{sign(w)}[b][i]
__global__ void __launch_bounds__(BP_BLOCK) k_bptt_dwin(BpttK k, BpttBwd g, int t)
{
    __shared__ unsigned long long s_mask[DWIN_J];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j0 = blockIdx.y * DWIN_J;
    const uint32_t* xw = k.x_bits + (size_t)t * k.B * k.Mw;
    for (int jj = warp; jj < DWIN_J; jj += BP_BLOCK / 32) {
        const int j = j0 + jj;
        const unsigned long long m = (j < k.M) ? trial_mask(xw, k.B, k.Mw, j, lane) : 0ull;
        if (lane == 0) s_mask[jj] = m;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k.N) return;
    for (int jj = 0; jj < DWIN_J; ++jj) {
        unsigned long long m = s_mask[jj];
        if (!m) continue;
        const size_t wi = (size_t)(j0 + jj) * k.N + i;
        const float w = k.w_in[wi];
        if (w == 0.0f) continue;
        const float* L = g.lamT + (w >= 0.0f ? 0 : (size_t)k.B * k.N) + i;
        float sum = 0.0f;
        while (m) {
            const int b = __ffsll((long long)m) - 1;
            m &= m - 1ull;
            sum += L[(size_t)b * k.N];
        }
        g.dw_in[wi] += sum;
    }
}

__global__ void k_bptt_fill_dense(const long long* rp, const int* col, const float* val, int N, float* dense)
{
    const int j = blockIdx.x;
    for (long long q = rp[j] + threadIdx.x; q < rp[j + 1]; q += blockDim.x) dense[(size_t)j * N + col[q]] = val[q];
}

__global__ void k_bptt_init(float* ymax, int* tmax, int n)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        ymax[q] = 0.0f;
        tmax[q] = 0;
    }
}

struct Work {
    size_t dense, Ie, Ii, v, y, u_seg, lam_u, lam_e, lam_i, lamS0, lamS1, lamT, R, ly0, ly1, colsel, total;
};

int bp_pad(int B) { return (B + 3) / 4 * 4; }

Work layout(const szsnn_bptt_desc* d)
{
    Work w{};
    const size_t BN = (size_t)d->B * d->N, BK = (size_t)d->B * d->K, NBp = (size_t)d->N * bp_pad(d->B);
    size_t o = 0;
    auto take = [&](size_t floats) { size_t r = o; o += (floats + 63) / 64 * 64; return r; };
    w.dense = take((size_t)d->N * d->N);
    w.Ie = take(BN); w.Ii = take(BN); w.v = take(BN); w.y = take(BK);
    w.u_seg = take((size_t)d->checkpoint_every * BN);
    w.lam_u = take(BN); w.lam_e = take(BN); w.lam_i = take(BN);
    w.lamS0 = take(2 * NBp); w.lamS1 = take(2 * NBp); w.lamT = take(4 * BN);
    w.R = take(NBp); w.ly0 = take(BK); w.ly1 = take(BK);
    w.colsel = take((size_t)d->nnz);  // ints, same size as floats
    w.total = o * sizeof(float);
    return w;
}

int check_desc(const szsnn_bptt_desc* d, char* err, size_t len)
{
    auto fail = [&](const char* m) {
        if (err && len) { std::strncpy(err, m, len - 1); err[len - 1] = 0; }
        return SZSNN_ERR_ARG;
    };
    if (!d) return fail("null descriptor");
    if (d->B < 1 || d->B > 64) return fail("batch must be 1..64");
    if (d->N < 1 || d->M < 1 || d->K < 1 || d->K > 64 || d->T < 1 || d->checkpoint_every < 1)
        return fail("bad sizes");
    if (d->tau_refrac != 0.0f) return fail("the adjoint supports tau_refrac == 0 only");
    if ((size_t)(d->M + d->N) * 4 > 200 * 1024) return fail("inputs + neurons exceed the shared-memory spike lists");
    if (d->N % 4) return fail("neurons must be a multiple of 4");
    return SZSNN_OK;
}

BpttK make_k(const szsnn_bptt_desc* d, float* ws)
{
    Work w = layout(d);
    BpttK k{};
    k.B = d->B; k.N = d->N; k.M = d->M; k.K = d->K; k.T = d->T; k.ck = d->checkpoint_every;
    k.Nw = (d->N + 31) / 32; k.Mw = (d->M + 31) / 32;
    k.v_rest = d->v_rest; k.cm = d->cm; k.tau_m = d->tau_m; k.i_offset = d->i_offset; k.v_reset = d->v_reset;
    k.v_thresh = d->v_thresh; k.alpha = d->alpha; k.beta = d->beta;
    k.de = sz_decay(d->tau_syn_E); k.di = sz_decay(d->tau_syn_I); k.km = sz_decay(d->tau_m);
    k.w_in = d->w_in; k.w_rec = ws + w.dense; k.rp = (const long long*)d->rec_row_ptr; k.col = d->rec_col;
    k.val = d->rec_val; k.w_out = d->w_out; k.x_bits = d->x_bits; k.spikes = d->spikes;
    k.Ie = ws + w.Ie; k.Ii = ws + w.Ii; k.v = ws + w.v; k.y = ws + w.y;
    k.ymax = d->ymax; k.tmax = d->tmax; k.vsum = d->vsum; k.u_seg = ws + w.u_seg; k.u_trace = d->u_trace;
    return k;
}

size_t step_smem(const szsnn_bptt_desc* d) { return (size_t)(d->M + d->N) * sizeof(int); }

}  // namespace

#define BP_TRY(x)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            if (err && err_len) { std::snprintf(err, err_len, "%s: %s", #x, cudaGetErrorString(e_)); } \
            return SZSNN_ERR_CUDA;                                                             \
        }                                                                                      \
    } while (0)

// Device time per phase, from CUDA events recorded on the stream between
// launches (only when the caller asks for it: it adds a synchronisation at the end).
struct PhaseTimer {
    double* out;
    cudaStream_t st;
    std::vector<cudaEvent_t> ev;
    std::vector<int> phase;
    PhaseTimer(double* o, cudaStream_t s) : out(o), st(s) {}
    ~PhaseTimer() { for (cudaEvent_t e : ev) cudaEventDestroy(e); }
    void mark(int ph)  // end of phase `ph` (-1: a start point)
    {
        if (!out) return;
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) { out = nullptr; return; }
        cudaEventRecord(e, st);
        ev.push_back(e);
        phase.push_back(ph);
    }
    cudaError_t finish()
    {
        if (!out || ev.empty()) return cudaSuccess;
        cudaError_t e = cudaEventSynchronize(ev.back());
        if (e != cudaSuccess) return e;
        for (size_t i = 1; i < ev.size(); ++i) {
            if (phase[i] < 0) continue;
            float ms = 0.0f;
            e = cudaEventElapsedTime(&ms, ev[i - 1], ev[i]);
            if (e != cudaSuccess) return e;
            out[phase[i]] += ms;
        }
        return cudaSuccess;
    }
};

extern "C" int szsnn_bptt_workspace_bytes(const szsnn_bptt_desc* d, uint64_t* bytes)
{
    if (!d || !bytes) return SZSNN_ERR_ARG;
    *bytes = layout(d).total;
    return SZSNN_OK;
}

extern "C" int szsnn_bptt_forward(const szsnn_bptt_desc* d, char* err, size_t err_len)
{
    int rc = check_desc(d, err, err_len);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)d->stream;
    float* ws = (float*)d->workspace;
    Work w = layout(d);
    BpttK k = make_k(d, ws);
    const size_t BN = (size_t)d->B * d->N;
    BP_TRY(cudaMemsetAsync(ws + w.dense, 0, (size_t)d->N * d->N * sizeof(float), st));
    k_bptt_fill_dense<<<d->N, 256, 0, st>>>(k.rp, k.col, k.val, d->N, ws + w.dense);
    BP_TRY(cudaGetLastError());
    BP_TRY(cudaMemsetAsync(k.Ie, 0, BN * 4, st));
    BP_TRY(cudaMemsetAsync(k.Ii, 0, BN * 4, st));
    BP_TRY(cudaMemcpyAsync(k.v, d->v0, BN * 4, cudaMemcpyDeviceToDevice, st));
    BP_TRY(cudaMemsetAsync(k.y, 0, (size_t)d->B * d->K * 4, st));
    BP_TRY(cudaMemsetAsync(d->vsum, 0, BN * 4, st));
    k_bptt_init<<<8, 256, 0, st>>>(d->ymax, d->tmax, d->B * d->K);
    BP_TRY(cudaGetLastError());
    const size_t smem = step_smem(d);
    BP_TRY(cudaFuncSetAttribute(k_bptt_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 1024)));
    const dim3 grid((unsigned)sz_div_up(d->N, BP_BLOCK * BP_NPT), (unsigned)d->B);
    for (int t = 0; t <= d->T; ++t) {
        if (t < d->T && t % d->checkpoint_every == 0) {
            float* c = d->ckpt + (size_t)(t / d->checkpoint_every) * 3 * BN;
            BP_TRY(cudaMemcpyAsync(c, k.Ie, BN * 4, cudaMemcpyDeviceToDevice, st));
            BP_TRY(cudaMemcpyAsync(c + BN, k.Ii, BN * 4, cudaMemcpyDeviceToDevice, st));
            BP_TRY(cudaMemcpyAsync(c + 2 * BN, k.v, BN * 4, cudaMemcpyDeviceToDevice, st));
        }
        k_bptt_step<<<grid, BP_BLOCK, smem, st>>>(k, t, 0, 0);
        BP_TRY(cudaGetLastError());
    }
    return SZSNN_OK;
}

extern "C" int szsnn_bptt_backward(const szsnn_bptt_desc* d, char* err, size_t err_len)
{
    int rc = check_desc(d, err, err_len);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)d->stream;
    float* ws = (float*)d->workspace;
    Work w = layout(d);
    BpttK k = make_k(d, ws);
    const size_t BN = (size_t)d->B * d->N, BK = (size_t)d->B * d->K;
    BpttBwd g{};
    const int Bp = bp_pad(d->B);
    const size_t NBp = (size_t)d->N * Bp;
    float* lamS[2] = {ws + w.lamS0, ws + w.lamS1};
    float* lamY[2] = {ws + w.ly0, ws + w.ly1};
    int* col_sel = reinterpret_cast<int*>(ws + w.colsel);
    g.lam_u = ws + w.lam_u; g.lam_e = ws + w.lam_e; g.lam_i = ws + w.lam_i;
    g.R = ws + w.R; g.col_sel = col_sel; g.Bp = Bp;
    g.g_ymax = d->g_ymax; g.g_vsum = d->g_vsum;
    g.dw_in = d->dw_in; g.dw_rec = d->dw_rec; g.dw_out = d->dw_out;
    for (float* p : {g.lam_u, g.lam_e, g.lam_i})
        BP_TRY(cudaMemsetAsync(p, 0, BN * 4, st));
    BP_TRY(cudaMemsetAsync(lamS[0], 0, 2 * NBp * 4, st));
    BP_TRY(cudaMemsetAsync(lamS[1], 0, 2 * NBp * 4, st));
    BP_TRY(cudaMemsetAsync(lamY[0], 0, BK * 4, st));
    BP_TRY(cudaMemsetAsync(lamY[1], 0, BK * 4, st));
    BP_TRY(cudaMemsetAsync(d->dw_in, 0, (size_t)d->M * d->N * 4, st));
    BP_TRY(cudaMemsetAsync(d->dw_rec, 0, (size_t)d->nnz * 4, st));
    BP_TRY(cudaMemsetAsync(d->dw_out, 0, (size_t)d->N * d->K * 4, st));
    if (d->nnz > 0) {
        k_bptt_colsel<<<1024, 256, 0, st>>>(k.col, k.val, d->nnz, d->N, col_sel);
        BP_TRY(cudaGetLastError());
    }
    const unsigned spmm_blocks = (unsigned)sz_div_up((int64_t)d->N * 32, BP_BLOCK);
    // optional per-phase device time (recompute, recurrent term + dWrec, adjoint, dWin)
    PhaseTimer pt(d->phase_ms, st);
    const size_t smem = step_smem(d);
    const dim3 grid_step((unsigned)sz_div_up(d->N, BP_BLOCK * BP_NPT), (unsigned)d->B);
    const dim3 grid((unsigned)sz_div_up(d->N, BP_BLOCK), (unsigned)d->B);
    const dim3 grid_in((unsigned)sz_div_up(d->N, BP_BLOCK), (unsigned)sz_div_up(d->M, DWIN_J));
    // The membrane trajectory the forward stored (u_trace, [T][B][N]) is one
    // segment read in place; otherwise each checkpoint segment is recomputed
    // into u_seg first (the same kernel, so the same u bit for bit).
    const bool stored = d->u_trace != nullptr;
    if (stored) k.u_seg = d->u_trace;
    const int seg_len = stored ? d->T : d->checkpoint_every;
    const int nseg = (d->T + seg_len - 1) / seg_len;
    // dWin(t) reads only lambda_t (lamT of t's parity), so it runs on a side
    // stream beside spmm(t-1); adjoint(t-2), which rewrites that parity half,
    // waits for it.  dW_in keeps its order of accumulation (t descending, one
    // stream).  With per-phase timing the phases stay on one stream.
    const bool side = d->phase_ms == nullptr;
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_lam[2] = {}, ev_dw[2] = {};
    struct Release {
        cudaStream_t* s; cudaEvent_t* a; cudaEvent_t* b;
        ~Release() { for (int p = 0; p < 2; ++p) { if (a[p]) cudaEventDestroy(a[p]); if (b[p]) cudaEventDestroy(b[p]); }
                     if (*s) cudaStreamDestroy(*s); }
    } release{&st2, ev_lam, ev_dw};
    if (side) {
        BP_TRY(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        for (int p = 0; p < 2; ++p) {
            BP_TRY(cudaEventCreateWithFlags(&ev_lam[p], cudaEventDisableTiming));
            BP_TRY(cudaEventCreateWithFlags(&ev_dw[p], cudaEventDisableTiming));
        }
        BP_TRY(cudaEventRecord(ev_dw[0], st));  // the side stream starts after the set-up above
        BP_TRY(cudaStreamWaitEvent(st2, ev_dw[0], 0));
    }
    bool dw_pending[2] = {false, false};
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int t0 = seg * seg_len, t1 = std::min(d->T, t0 + seg_len);
        if (!stored) {
            const float* c = d->ckpt + (size_t)seg * 3 * BN;
            BP_TRY(cudaMemcpyAsync(k.Ie, c, BN * 4, cudaMemcpyDeviceToDevice, st));
            BP_TRY(cudaMemcpyAsync(k.Ii, c + BN, BN * 4, cudaMemcpyDeviceToDevice, st));
            BP_TRY(cudaMemcpyAsync(k.v, c + 2 * BN, BN * 4, cudaMemcpyDeviceToDevice, st));
            pt.mark(-1);
            for (int t = t0; t < t1; ++t) {  // recompute u_t from the checkpoint, spikes kept
                k_bptt_step<<<grid_step, BP_BLOCK, smem, st>>>(k, t, 1, t0);
                BP_TRY(cudaGetLastError());
            }
            pt.mark(0);
        } else {
            pt.mark(-1);
        }
        for (int t = t1 - 1; t >= t0; --t) {
            const int par = t & 1;  // buffers of step t; step t+1 uses the other parity
            const bool have_R = t < d->T - 1;
            if (have_R) {  // R from lambda_{t+1}, and dWrec of step t+1 (spikes of step t)
                k_bptt_spmm<<<spmm_blocks, BP_BLOCK, 0, st>>>(k, col_sel, Bp, lamS[par ^ 1], ws + w.R, d->dw_rec, t);
                BP_TRY(cudaGetLastError());
            }
            pt.mark(1);
            g.lamS = lamS[par];
            g.lam_y = lamY[par];
            g.lam_y_next = lamY[par ^ 1];
            g.lamT = ws + w.lamT + (size_t)par * 2 * BN;
            if (dw_pending[par]) BP_TRY(cudaStreamWaitEvent(st, ev_dw[par], 0));  // dWin(t+2) done with this half
            k_bptt_adjoint<<<grid, BP_BLOCK, 0, st>>>(k, g, t, t0, have_R ? 1 : 0);
            BP_TRY(cudaGetLastError());
            pt.mark(2);
            if (side) {
                BP_TRY(cudaEventRecord(ev_lam[par], st));
                BP_TRY(cudaStreamWaitEvent(st2, ev_lam[par], 0));
                k_bptt_dwin<<<grid_in, BP_BLOCK, 0, st2>>>(k, g, t);
                BP_TRY(cudaGetLastError());
                BP_TRY(cudaEventRecord(ev_dw[par], st2));
                dw_pending[par] = true;
            } else {
                k_bptt_dwin<<<grid_in, BP_BLOCK, 0, st>>>(k, g, t);
                BP_TRY(cudaGetLastError());
            }
            pt.mark(3);
        }
    }
    if (side) {  // the caller's stream resumes after the last dWin
        BP_TRY(cudaEventRecord(ev_dw[0], st2));
        BP_TRY(cudaStreamWaitEvent(st, ev_dw[0], 0));
    }
    BP_TRY(pt.finish());
    return SZSNN_OK;
}
