// net.cu -- native B200 network path.
//
// Design (replaces the reference's bundle/queue layout, which cannot hold a
// 1e9-synapse network: GroupData.cpp:94 sizes groupPtrs for every
// (neuron, delay) pair and pads every bundle to 32 slots):
//  * synapses: one row per unit (neurons, then sources), each row bucketed by
//    delay m = 1..D; interleaved {int32 target, fp32 weight} = 8 B per synapse
//    (the delay is implied by the bucket);
//  * spike ring: D+1 slots of compacted spike ids.  Step t's update appends to
//    slot t % (D+1); step t's propagate delivers slot (t-m) % (D+1) over
//    bucket m for m = 1..D.  This is the reference's per-delay ring
//    (scatter_kernel.cl:154) with the fan-out done at delivery time, so the
//    accumulation targets the current step's 2 x N input arrays only
//    (L2-resident: 8 MB at N = 1e6);
//  * propagate: grid-stride over (m, spike) work items, G lanes per bucket
//    segment, fp32 `red` atomics into in_exc / in_inh split by weight sign
//    (gather_kernel.cl:172-178), or int64 fixed-point atomics for
//    bit-reproducible sums;
//  * update: one thread per unit for neurons and sources (Poisson draws from
//    Philox), consuming and clearing the inputs, spikes compacted with a warp
//    ballot and one atomic per spiking warp, raster word written from the
//    ballot;
//  * steps captured in CUDA graphs of `chunk` steps; the step counter lives in
//    device memory, so no host synchronisation happens between steps;
//  * overlapped stepping (default): the input arrays are double-buffered by
//    step parity.  Delivery of delays m >= 2 into step t+1's inputs only
//    reads ring slots of steps <= t-1, so it runs on a second stream while
//    update(t) runs; update(t) itself delivers the m = 1 bucket of the units
//    that spike in it (one warp per spiking warp).  The classic order
//    (propagate(t) with m = 1..D, then update(t), one buffer) remains
//    selectable and is what the allocation-free single step uses.
#include "common.cuh"

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

// slots 0..11 as szsnn_pop_desc; 12, 13 = 1 - 1/tau_syn_E, 1 - 1/tau_syn_I
// (IF models), computed once on the host with the same fp32 operations
#define POP_SLOTS 16
#define INLINE_POPS 4
#define UPD_UPT 4        // units per update thread chosen by default (strided by the block size)
#define UPD_MAX_UPT 16   // most units per update thread szsnn_net_set_update_units accepts
#define UPD_MAX_BLOCK 256  // update threads per block (the step kernel's block too)
#define UPD_MIN_BLOCKS 6   // resident blocks of UPD_MAX_BLOCK per SM the register budget keeps
struct PopDev {
    int32_t model;
    uint32_t flags;
    int64_t begin, end;
    float p[POP_SLOTS];
    const float* pn;   // per-unit parameters [POP_SLOTS][end-begin], or null
    uint64_t seed;
};

struct NetDev {
    int64_t N, U, words;
    int32_t D, npops;
    const PopDev* pops;
    const unsigned long long* row_ptr;
    const unsigned long long* rp_dm;  // delay-major copy: rp_dm[m * U + u] = row_ptr[u * D + m], m = 0..D; or null
    const int2* syn;
    float* st0;
    float* st1;
    float* st2;
    float* st3;
    float* in_e;          // parity-0 input buffers (the only ones in classic order)
    float* in_i;
    long long* fx_e;
    long long* fx_i;
    float* in_e1;         // parity-1 buffers (overlapped stepping)
    float* in_i1;
    long long* fx_e1;
    long long* fx_i1;
    uint32_t overlap;
    uint32_t acc_mode;
    uint32_t* ring_cnt;
    int32_t* ring_ids;
    const long long* clock;
    unsigned long long* stats;  // [0] events consumed, [1] spikes (all but the newest step),
                                // [2 + p] events delivered into the parity-p buffer, not yet consumed
    uint32_t* err;
    float* dbg_in_e;
    float* dbg_in_i;
    const int32_t* group;                  // per-unit group or null
    unsigned long long* group_spikes;      // [n_groups]
    const int2* blk_pop;                   // per update block: (first overlapping pop, count)
    uint32_t par0;                         // parity of the step counter when the launch runs
    int32_t upt;                           // units per update thread (1..UPD_MAX_UPT)
    int32_t ib_lo[INLINE_POPS], ib_hi[INLINE_POPS];  // update blocks [lo, hi) lying inside slot i (empty: none)
    PopDev ipop[INLINE_POPS];              // populations with shared parameters, by value in the kernel parameters
    uint32_t tiles;                        // update tile scheme: 0 a block per tile, 1 persistent warp tiles,
                                           // 2 persistent block tiles
    int64_t own_lo[2], own_hi[2];          // units this network updates: neurons [0], sources [1]
};

// the unit is updated here (a sharded network updates its own ranges only)
__device__ __forceinline__ bool owned(const NetDev& nd, int64_t id)
{
    return (id >= nd.own_lo[0] && id < nd.own_hi[0]) || (id >= nd.own_lo[1] && id < nd.own_hi[1]);
}

struct szsnn_net {
    szsnn_ctx* ctx = nullptr;
    int64_t N = 0, U = 0, words = 0;
    int32_t D = 0, R = 0;
    uint32_t acc_mode = 0;
    int32_t npops = 0;
    std::vector<szsnn_pop_desc> pops;
    PopDev* d_pops = nullptr;
    std::vector<PopDev> h_pops;            // the device table's host copy (kernel-parameter table)
    float* d_pn = nullptr;                 // all per-unit parameter arrays, back to back
    int32_t* d_group = nullptr;
    unsigned long long* d_group_spikes = nullptr;
    int32_t n_groups = 0;
    // state monitor: recorded slots of chosen units, appended on the device after every step
    int32_t* d_mon_ids = nullptr;
    int32_t mon_n = 0;                     // monitored units (0: off)
    uint32_t mon_slots = 0;                // bit k: state slot k recorded
    float* d_mon_buf = nullptr;            // [capacity][slots][units]
    long long* d_mon_t0 = nullptr;         // the step the trace starts at (device copy)
    int64_t mon_cap = 0, mon_t0 = 0;
    int2* d_blk_pop = nullptr;             // per update-block tile: sized for 32-thread blocks, filled for upd_block
    uint64_t n_syn = 0;
    unsigned long long* d_row_ptr = nullptr;
    unsigned long long* d_rp_dm = nullptr;     // delay-major copy of the bucket starts (delivery reads)
    int2* d_syn = nullptr;
    float* d_st[4] = {};
    float* d_in_e[2] = {};       // exc / inh inputs, one buffer per step parity (overlapped stepping)
    float* d_in_i[2] = {};
    long long* d_fx_e[2] = {};   // fixed-point inputs (acc_mode FIXED)
    long long* d_fx_i[2] = {};
    uint32_t* d_ring_cnt = nullptr;
    int32_t* d_ring_ids = nullptr;
    long long* d_clock = nullptr;
    unsigned long long* d_stats = nullptr;
    int chunk = 100;
    uint32_t* d_forced_stage[2] = {};   // chunk * words each, alternating chunks
    float* d_current_stage = nullptr;
    uint32_t* d_raster_stage[2] = {};
    float* d_dbg_in = nullptr;
    uint32_t* h_pinned_words = nullptr;  // pinned: one step's words (szsnn_net_step)
    uint32_t* d_inject = nullptr;        // spike words of other shards (szsnn_net_inject_spikes)
    uint32_t* h_io[4] = {};              // pinned bounce buffers for pageable host arrays: in0, in1, out0, out1
    cudaStream_t copy_st = nullptr;      // host -> device copies of szsnn_net_run (forced words)
    cudaStream_t copy_out_st = nullptr;  // device -> host copies of szsnn_net_run (raster)
    cudaEvent_t ev_in[2] = {}, ev_comp[2] = {}, ev_out[2] = {};
    bool overlap = true;
    std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> graphs;  // (steps, io flags, stage, step parity)
    int64_t steps_done = 0;
    uint64_t graph_launches = 0, kernel_launches = 0;
    int prop_mode = 0, prop_group = 16, prop_blocks = 0, upd_block = 256;
    int upd_tiles = 0, upd_per_sm = 0;   // update tiles: 0 block tiles, 1 persistent warp tiles (blocks per SM)
    int upd_units = 0;                   // units per update thread (0: automatic, upd_upt)
    int64_t own_lo[2] = {0, 0}, own_hi[2] = {-1, -1};  // owned neuron / source ranges (-1: all)
    double t_prop_ms = 0, t_upd_ms = 0, t_total_ms = 0;
    cudaEvent_t ev_run0 = nullptr, ev_run1 = nullptr;  // around the last szsnn_net_run*
    bool run_timed = false;
    // resident stepping: one cooperative launch per chunk, neuron state in shared memory
    bool resident = false;
    int res_uw = 16, res_blocks = 0;     // update warps per block, blocks (0: one per SM)
    unsigned int* d_res_sync = nullptr;  // grid-barrier arrivals and abort flag
};

namespace {

struct UnitParams {  // per-unit parameter arrays
    const float* pn;
    int64_t off, cnt;
    __device__ __forceinline__ float operator()(int k) const { return pn[(int64_t)k * cnt + off]; }
};
struct SharedParams {  // one parameter set for the population (staged in shared memory)
    const float* p;
    __device__ __forceinline__ float operator()(int k) const { return p[k]; }
};

// neuron update for one unit; returns the spike
template <class P>
__device__ __forceinline__ bool run_neuron(const P& p, int model, uint32_t flags, float& v, float& g1, float& g2,
                                           float& fr, float in_e, float in_i, float i_ext, bool f)
{
    if (model == SZSNN_IF_CURR_EXP) return sz_if_curr_exp(p, v, g1, g2, fr, in_e, in_i, i_ext, f, p(12), p(13));
    if (model == SZSNN_IF_COND_EXP) return sz_if_cond_exp(p, v, g1, g2, fr, in_e, in_i, i_ext, f, p(12), p(13));
    if (model == SZSNN_IZHIKEVICH)
        return sz_izhikevich(p, v, g1, in_e, in_i, i_ext, f, (flags & SZSNN_POP_IZH_HALF_STEPS) != 0);
    return false;
}

__global__ void k_advance(long long* clock, int k) { *clock += k; }

// State monitor: after step t (= step counter + k_off) the recorded slots of
// the monitored units go to row t - t0 of the trace, when it fits.
__global__ void k_monitor(const long long* __restrict__ clock, int k_off, const long long* __restrict__ t0,
                          const float* __restrict__ st0, const float* __restrict__ st1,
                          const float* __restrict__ st2, const float* __restrict__ st3,
                          const int32_t* __restrict__ ids, int n, uint32_t slots, float* __restrict__ buf,
                          long long cap)
{
    const long long r = *clock + k_off - *t0;
    if (r < 0 || r >= cap) return;
    const int ns = __popc(slots);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t u = ids[i];
        int j = 0;
        if (slots & 1u) buf[((size_t)r * ns + j++) * n + i] = st0[u];
        if (slots & 2u) buf[((size_t)r * ns + j++) * n + i] = st1[u];
        if (slots & 4u) buf[((size_t)r * ns + j++) * n + i] = st2[u];
        if (slots & 8u) buf[((size_t)r * ns + j++) * n + i] = st3[u];
    }
}

// propagate flags
#define PF_ZERO_SLOT 1u  // zero the ring count of slot t (classic order: update(t) fills it next)
#define PF_SPIKES 2u     // add the spike count of step t-1 to the statistics
#define PF_PENDING 4u    // count events as delivered into the parity buffer of step t, not yet consumed

struct InBuf {
    float* e;
    float* i;
    long long* fe;
    long long* fi;
};

// input buffers that step t's update consumes
__device__ __forceinline__ InBuf in_buf(const NetDev& nd, long long t)
{
    if (nd.overlap && (t & 1)) return InBuf{nd.in_e1, nd.in_i1, nd.fx_e1, nd.fx_i1};
    return InBuf{nd.in_e, nd.in_i, nd.fx_e, nd.fx_i};
}

// the same buffers from the host-known parity (no wait for the step counter)
__device__ __forceinline__ InBuf in_buf_k(const NetDev& nd, int k_off)
{
    return in_buf(nd, (long long)((nd.par0 + (uint32_t)k_off) & 1u));
}

// bounds [a, e) of bucket m (delay m, 1-based) of unit u, from the
// delay-major copy (dm: warp-uniform; the warp's units are mostly consecutive,
// so their bucket starts share sectors there) or from the unit-major row_ptr
// (scattered units: both bounds of a bucket in one sector)
__device__ __forceinline__ void bucket_bounds(const NetDev& nd, bool dm, int64_t u, int m, unsigned long long& a,
                                              unsigned long long& e)
{
    if (dm) {
        a = __ldg(&nd.rp_dm[(int64_t)(m - 1) * nd.U + u]);
        e = __ldg(&nd.rp_dm[(int64_t)m * nd.U + u]);
    } else {
        a = __ldg(&nd.row_ptr[u * nd.D + (m - 1)]);
        e = __ldg(&nd.row_ptr[u * nd.D + m]);
    }
}

// one synapse into the exc / inh input of its target (weight sign picks the
// channel, gather_kernel.cl:172-178; w == 0 is padding and counts nothing)
__device__ __forceinline__ void deliver(const NetDev& nd, const InBuf& b, int2 sw, uint32_t& ev)
{
    const float w = __int_as_float(sw.y);
    if (w == 0.0f) return;
    if ((unsigned long long)sw.x >= (unsigned long long)nd.N) {
        dev_error(nd.err, SZSNN_DEV_BAD_TARGET, (uint32_t)sw.x);
        return;
    }
    ++ev;
    if (nd.acc_mode == SZSNN_ACC_FIXED) {
        const long long qv = __float2ll_rn(w * 4294967296.0f);
        atomicAdd((unsigned long long*)(w >= 0.0f ? &b.fe[sw.x] : &b.fi[sw.x]), (unsigned long long)qv);
    } else {
        atomicAdd(w >= 0.0f ? &b.e[sw.x] : &b.i[sw.x], w);
    }
}

// ring-slot counts of delays m_lo..D for step t, inclusive scan in s_pre[1..D]
// (s_pre[0] = 0); block 0 does the slot / statistics bookkeeping of `pf`
__device__ __forceinline__ void propagate_prologue(const NetDev& nd, long long t, int m_lo, uint32_t pf,
                                                   uint32_t* s_pre, unsigned long long* s_ev, bool lead)
{
    const int D = nd.D, R = D + 1;
    for (int m = threadIdx.x + 1; m <= D; m += blockDim.x) {
        const long long tm = t - m;
        s_pre[m] = (m >= m_lo && tm >= 0) ? nd.ring_cnt[tm % R] : 0u;
    }
    if (threadIdx.x == 0) { s_pre[0] = 0; *s_ev = 0; }
    __syncthreads();
    if (threadIdx.x < 32) {  // inclusive scan of counts over m = 1..D
        uint32_t carry = 0;
        const uint32_t lane = threadIdx.x;
        for (int m0 = 1; m0 <= D; m0 += 32) {
            const int m = m0 + (int)lane;
            const uint32_t c = (m <= D) ? s_pre[m] : 0u;
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += y;
            }
            if (m <= D) s_pre[m] = carry + incl;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
    if (lead && threadIdx.x == 0) {
        if (pf & PF_ZERO_SLOT) nd.ring_cnt[t % R] = 0;  // slot t held step t-R, no longer needed
        if ((pf & PF_SPIKES) && t >= 1) atomicAdd(&nd.stats[1], (unsigned long long)s_pre[1]);  // step t-1
    }
}

__device__ __forceinline__ void propagate_epilogue(const NetDev& nd, long long t, uint32_t pf, uint32_t ev,
                                                   unsigned long long* s_ev)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ev += __shfl_down_sync(0xffffffffu, ev, o);
    if ((threadIdx.x & 31) == 0 && ev) atomicAdd(s_ev, (unsigned long long)ev);
    __syncthreads();
    if (threadIdx.x == 0 && *s_ev) atomicAdd(&nd.stats[(pf & PF_PENDING) ? 2 + (t & 1) : 0], *s_ev);
}

// Delivery of ring slots t-m, m = m_lo..D, over bucket m of each spiking unit
// into step t's inputs: grid-stride over (delay, spike) work items, G lanes
// per bucket segment.
// (blk, nblk): this block's index among the nblk blocks doing the delivery
template <int G>
__device__ __forceinline__ void propagate_grouped(const NetDev& nd, int k_off, int m_lo, uint32_t pf, int blk, int nblk)
{
    __shared__ uint32_t s_pre[1025];
    __shared__ unsigned long long s_ev;
    const long long t = *nd.clock + k_off;
    const int D = nd.D, R = D + 1;
    propagate_prologue(nd, t, m_lo, pf, s_pre, &s_ev, blk == 0);
    const InBuf buf = in_buf(nd, t);
    const uint32_t total = s_pre[D];
    const uint32_t lg = threadIdx.x % G;
    const int64_t gid = ((int64_t)blk * blockDim.x + threadIdx.x) / G;
    const int64_t ngroups = ((int64_t)nblk * blockDim.x) / G;
    uint32_t ev = 0;
    for (int64_t item = gid; item < (int64_t)total; item += ngroups) {
        int lo = 1, hi = D;  // first m with s_pre[m] > item
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int64_t)s_pre[mid] > item) hi = mid; else lo = mid + 1;
        }
        const int m = lo;
        const uint32_t j = (uint32_t)(item - s_pre[m - 1]);
        const int64_t slot = (t - m) % R;
        const int64_t s = nd.ring_ids[slot * nd.U + j];
        unsigned long long a, e;
        bucket_bounds(nd, false, s, m, a, e);
        for (unsigned long long q = a + lg; q < e; q += G) deliver(nd, buf, nd.syn[q], ev);
    }
    propagate_epilogue(nd, t, pf, ev, &s_ev);
}

template <int G>
__global__ void __launch_bounds__(256) k_propagate(const __grid_constant__ NetDev nd, int k_off, int m_lo, uint32_t pf)
{
    propagate_grouped<G>(nd, k_off, m_lo, pf, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 8-byte asynchronous copy global -> shared (no register holds the data in
// flight); completed by cp_async_wait_all in the issuing thread
__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(smem_addr(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Synapses in flight per lane of a delivery warp, and the shared-memory
// window that holds them: 32 * FAR_WPL int2 per warp
#define FAR_WPL 12
__host__ __device__ __forceinline__ size_t far_window_bytes(int block_threads)
{
    return (size_t)(block_threads / 32) * 32 * FAR_WPL * sizeof(int2);
}

// The warp's share of the flattened items of step t (s_pre: the scan of
// the ring counts by delay): warp gw of nw takes items gw * IPW + k * nw * IPW
// onward.  Returns the synapses it delivered.  CG: ring ids read through L2
// only (a launch that also appends to the ring it reads).
template <int IPW, bool CG>
__device__ __forceinline__ uint32_t flat_items(const NetDev& nd, long long t, const uint32_t* s_pre, int64_t gw,
                                               int64_t nw, int2* win, const InBuf& buf)
{
    const int D = nd.D, R = D + 1;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t total = s_pre[D];
    const int2* __restrict__ syn = nd.syn;
    uint32_t ev = 0;
    for (int64_t base = gw * IPW; base < (int64_t)total; base += nw * IPW) {
        const int64_t item = base + lane;
        unsigned long long a = 0, e = 0;
        int64_t s = -1;
        int mm = 0;  // the item's delay, 0 for lanes without one
        if (lane < (uint32_t)IPW && item < (int64_t)total) {
            int lo = 1, hi = D;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if ((int64_t)s_pre[mid] > item) hi = mid; else lo = mid + 1;
            }
            const int m = lo;
            const uint32_t j = (uint32_t)(item - s_pre[m - 1]);
            const int32_t* rid = &nd.ring_ids[((t - m) % R) * nd.U + j];
            s = CG ? __ldcg(rid) : __ldg(rid);
            mm = m;
        }
        // the delay-major index when most of the warp's items are consecutive
        // units at one delay (a ring slot of a warp-wide burst), else row_ptr
        const int64_t s_prev = __shfl_up_sync(0xffffffffu, s, 1);
        const int m_prev = __shfl_up_sync(0xffffffffu, mm, 1);
        const bool consec = lane > 0 && mm > 0 && m_prev == mm && s == s_prev + 1;
        const bool dm = nd.rp_dm && __popc(__ballot_sync(0xffffffffu, consec)) >= IPW / 2;
        if (mm > 0) bucket_bounds(nd, dm, s, mm, a, e);
        const uint32_t len = (uint32_t)(e - a);
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        const uint32_t excl = incl - len;
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        // window [k0, k0 + W) of the concatenation: each item lane copies the
        // part of its own segment inside the window to its place in the
        // warp's slice, waits for its copies, and after a warp barrier every
        // lane delivers W / 32 entries of the window
        constexpr uint32_t W = 32 * FAR_WPL;
        for (uint32_t k0 = 0; k0 < tot; k0 += W) {
            const uint32_t j0 = k0 > excl ? k0 - excl : 0u;
            const uint32_t j1 = min(len, k0 + W - min(k0 + W, excl));
            for (uint32_t j = j0; j < j1; ++j) cp_async8(&win[excl + j - k0], &syn[a + j]);
            cp_async_wait_all();
            __syncwarp();
#pragma unroll
            for (int u = 0; u < FAR_WPL; ++u)
                if (k0 + 32u * u + lane < tot) deliver(nd, buf, win[32 * u + lane], ev);
            __syncwarp();
        }
    }
    return ev;
}

// Warp-flattened delivery: lanes 0..IPW-1 each resolve one (delay, spike)
// work item to its bucket segment; the warp then walks the concatenation of
// those segments in windows of 32 * FAR_WPL synapses.  Each item lane issues
// asynchronous 8-byte copies of its segment's part of the window into the
// warp's shared-memory slice and waits for them; after a warp barrier every
// lane delivers FAR_WPL entries of the window: one memory round trip per
// window rather than one per few loads, with no registers holding the loads
// in flight.
// Dynamic shared memory: far_window_bytes(blockDim.x).
template <int IPW>
__device__ __forceinline__ void propagate_flat(const NetDev& nd, int k_off, int m_lo, uint32_t pf, int blk, int nblk)
{
    __shared__ uint32_t s_pre[1025];
    __shared__ unsigned long long s_ev;
    extern __shared__ __align__(128) unsigned char upd_smem[];
    const long long t = *nd.clock + k_off;
    propagate_prologue(nd, t, m_lo, pf, s_pre, &s_ev, blk == 0);
    const InBuf buf = in_buf(nd, t);
    const int64_t gw = ((int64_t)blk * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)nblk * blockDim.x) >> 5;
    int2* const win = reinterpret_cast<int2*>(upd_smem) + (size_t)(threadIdx.x >> 5) * 32 * FAR_WPL;
    const uint32_t ev = flat_items<IPW, false>(nd, t, s_pre, gw, nw, win, buf);
    propagate_epilogue(nd, t, pf, ev, &s_ev);
}

template <int IPW>
__global__ void __launch_bounds__(256, 4) k_propagate_flat(const __grid_constant__ NetDev nd, int k_off, int m_lo, uint32_t pf)
{
    propagate_flat<IPW>(nd, k_off, m_lo, pf, blockIdx.x, gridDim.x);
}

// last population with begin <= id, or -1 (ranges sorted and disjoint)
__device__ __forceinline__ int find_pop(const PopDev* pops, int npops, int64_t id)
{
    int pi = -1;
    for (int lo = 0, hi = npops - 1; lo <= hi;) {
        const int mid = (lo + hi) >> 1;
        if (pops[mid].begin <= id) { pi = mid; lo = mid + 1; } else hi = mid - 1;
    }
    return pi;
}

#define UPD_BLOCK_POPS 8

// Spike bookkeeping of one warp: group counters, raster word, compaction into
// ring slot t (one atomic per spiking warp) and, in the overlapped order,
// delivery of the spiking units' delay-1 buckets into step t+1's inputs.
__device__ __forceinline__ void update_spikes(const NetDev& nd, long long t, int64_t id, bool spk, uint32_t lane,
                                              uint32_t* __restrict__ out_words)
{
    if (spk && nd.group) atomicAdd(&nd.group_spikes[nd.group[id]], 1ull);
    const uint32_t ball = __ballot_sync(0xffffffffu, spk);
    const int64_t wd = id >> 5;
    if (lane == 0 && out_words && wd < nd.words) out_words[wd] = ball;
    if (ball) {
        // the delay-1 bucket bounds are loaded before the ring append, so the
        // two round trips overlap
        unsigned long long ra = 0, re = 0;
        if (nd.overlap && spk) bucket_bounds(nd, nd.rp_dm && __popc(ball) >= 8, id, 1, ra, re);
        const int R = nd.D + 1;
        const int64_t slot = t % R;
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&nd.ring_cnt[slot], (uint32_t)__popc(ball));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (spk) {
            uint32_t rank = __popc(ball & ((1u << lane) - 1u));
            uint32_t pos = base + rank;
            if (pos < (uint32_t)nd.U) nd.ring_ids[slot * nd.U + pos] = (int32_t)id;
            else dev_error(nd.err, SZSNN_DEV_RING_OVERFLOW, (uint32_t)slot);
        }
        if (nd.overlap) {  // m = 1 buckets of this warp's spiking units into step t+1's inputs
            // one walk over the concatenated buckets, 32 synapses per pass (owner
            // lane by a search over the exclusive offsets), NEAR_UNR loads in
            // flight per lane, so a warp of many spiking units pays a few round
            // trips rather than one per unit
            constexpr int NEAR_UNR = 2;
            const InBuf nb = in_buf(nd, t + 1);
            const uint32_t len = (uint32_t)(re - ra);
            uint32_t incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += y;
            }
            const uint32_t excl = incl - len;
            const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
            uint32_t ev = 0;
            for (uint32_t k0 = 0; k0 < tot; k0 += 32 * NEAR_UNR) {
                int2 sw[NEAR_UNR];
                bool ok[NEAR_UNR];
#pragma unroll
                for (int u = 0; u < NEAR_UNR; ++u) {
                    const uint32_t k = k0 + 32u * u + lane;
                    ok[u] = k < tot;
                    int owner = 0;  // last lane whose segment starts at or before k
#pragma unroll
                    for (int st = 16; st >= 1; st >>= 1) {
                        const int cand = owner + st;
                        const uint32_t ex = __shfl_sync(0xffffffffu, excl, cand & 31);
                        if (cand < 32 && ex <= k) owner = cand;
                    }
                    const unsigned long long oa = __shfl_sync(0xffffffffu, ra, owner);
                    const uint32_t oex = __shfl_sync(0xffffffffu, excl, owner);
                    sw[u] = ok[u] ? nd.syn[oa + (k - oex)] : make_int2(0, 0);
                }
#pragma unroll
                for (int u = 0; u < NEAR_UNR; ++u)
                    if (ok[u]) deliver(nd, nb, sw[u], ev);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ev += __shfl_down_sync(0xffffffffu, ev, o);
            if (lane == 0 && ev) atomicAdd(&nd.stats[2 + ((t + 1) & 1)], (unsigned long long)ev);
        }
    }
}

// Per-step bookkeeping of the overlapped order, by one thread of update block
// 0: spikes of step t-1 into the statistics, ring slot t+1 emptied for
// update(t+1) (it held step t-D, read last by the delivery into step t),
// events of step t's buffer moved from pending to consumed.
__device__ __forceinline__ void step_bookkeeping(const NetDev& nd, long long t)
{
    // L2 loads: a resident launch reads counters other blocks wrote in it
    const int R = nd.D + 1;
    if (t >= 1) atomicAdd(&nd.stats[1], (unsigned long long)__ldcg(&nd.ring_cnt[(t - 1) % R]));
    nd.ring_cnt[(t + 1) % R] = 0;
    const unsigned long long pend = __ldcg(&nd.stats[2 + (t & 1)]);
    nd.stats[2 + (t & 1)] = 0;
    atomicAdd(&nd.stats[0], pend);
}

// Unit state and inputs of the generic update, loaded before the block's
// population lookup so the loads of a warp are in flight together.
struct UnitIn {
    float v, g1, g2, fr, in_e, in_i, i_ext;
    long long fxe, fxi;
    bool f;
};

// ---- inline tiles: blocks inside one population of the parameter table
//
// The block's tile of T = nd.upt * blockDim.x units is brought into shared
// memory by bulk copies (one per state / input array, issued by one thread,
// completing on an mbarrier), so the bytes in flight are bounded by shared
// memory rather than by registers.  Each thread then updates units
// j * blockDim.x + threadIdx.x of the tile from shared memory, with the
// population's parameters as constant-bank operands (slot and model
// compile-time), writing the new state and the cleared inputs back into
// the tile; after the last sub-tile one bulk store per array returns the
// tile to global memory.
// Dynamic shared memory: mbarrier at 0, arrays from byte 16: st0..st3 (T
// floats each), then the exc / inh inputs (T floats or T int64 each).
__host__ __device__ __forceinline__ size_t tile_smem_bytes(int64_t T, bool fixed)
{
    return 16 + (size_t)T * (16 + (fixed ? 16 : 8));
}

struct TileSmem {
    uint64_t* bar;
    float* st[4];
    float* ie;
    float* ii;
    long long* fe;
    long long* fi;
};

__device__ __forceinline__ TileSmem tile_smem(unsigned char* base, uint32_t T, bool fixed)
{
    TileSmem m;
    m.bar = reinterpret_cast<uint64_t*>(base);
    float* f = reinterpret_cast<float*>(base + 16);
    for (int k = 0; k < 4; ++k) m.st[k] = f + (size_t)k * T;
    m.ie = f + 4 * (size_t)T;
    m.ii = f + 5 * (size_t)T;
    m.fe = reinterpret_cast<long long*>(f + 4 * (size_t)T);
    m.fi = m.fe + T;
    return m;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 :: "l"(dst), "r"(smem_addr(src)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// the issuing thread's bulk stores have read their shared-memory sources
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0u;
}

// bounded wait for the phase of the tile's mbarrier with parity `parity`
__device__ __forceinline__ bool tile_wait(uint64_t* bar, uint32_t parity = 0u)
{
    for (int i = 0; i < (1 << 20); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Issue the tile's bulk copies (thread 0) and wait for them (all threads).
// Model M decides which arrays a unit reads; Poisson tiles read none.
// phase < 0: a block with one tile (the mbarrier is initialised here and its
// phase 0 awaited); phase >= 0: a persistent block whose mbarrier was
// initialised once, awaiting the phase of this tile's parity.
template <int MODEL, bool FIXED>
__device__ __forceinline__ bool tile_load(const NetDev& nd, const InBuf& inb, int64_t tile0, uint32_t T,
                                          const TileSmem& sm, int phase = -1)
{
    if (MODEL == SZSNN_POISSON) return true;
    if (threadIdx.x == 0) {  // init, then the copies at once; the block barrier below orders the waits after the init
        if (phase < 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(sm.bar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        const int64_t n = min((int64_t)T, nd.U - tile0);  // the tile lies inside a neuron population
        const uint32_t b4 = (uint32_t)((n * 4 + 15) & ~(int64_t)15);
        const uint32_t b8 = (uint32_t)((n * 8 + 15) & ~(int64_t)15);
        const int nst = MODEL == SZSNN_IZHIKEVICH ? 2 : 4;
        const uint32_t total = (uint32_t)nst * b4 + 2u * (FIXED ? b8 : b4);
        asm volatile("{\n .reg .b64 s;\n mbarrier.arrive.expect_tx.shared::cta.b64 s, [%0], %1;\n}"
                     :: "r"(smem_addr(sm.bar)), "r"(total) : "memory");
        float* const gst[4] = {nd.st0, nd.st1, nd.st2, nd.st3};
        for (int k = 0; k < nst; ++k) bulk_load(sm.st[k], gst[k] + tile0, b4, sm.bar);
        if (FIXED) {
            bulk_load(sm.fe, inb.fe + tile0, b8, sm.bar);
            bulk_load(sm.fi, inb.fi + tile0, b8, sm.bar);
        } else {
            bulk_load(sm.ie, inb.e + tile0, b4, sm.bar);
            bulk_load(sm.ii, inb.i + tile0, b4, sm.bar);
        }
    }
    __syncthreads();
    const uint32_t parity = phase < 0 ? 0u : (uint32_t)(phase & 1);
    if (tile_wait(sm.bar, parity)) return true;
    // the copies did not complete in time: report, wait once more so none is
    // still writing shared memory when the block leaves, skip the tile
    if (threadIdx.x == 0) dev_error(nd.err, SZSNN_DEV_WAIT_TIMEOUT, (uint32_t)tile0);
    tile_wait(sm.bar, parity);
    return false;
}

// one unit of an inline tile, from shared memory (u = index in the tile)
template <int MODEL, bool FIXED>
__device__ __forceinline__ bool tile_unit(const NetDev& nd, const PopDev& P, const InBuf& inb, const TileSmem& sm,
                                          uint32_t id, uint32_t u, long long t, const uint32_t* __restrict__ forced,
                                          const float* __restrict__ current)
{
    const bool f = forced ? ((forced[id >> 5] >> (id & 31)) & 1u) != 0u : false;
    if (MODEL == SZSNN_POISSON) return sz_poisson_fires(P.seed, (int64_t)id - P.begin, t, P.p[0]) || f;
    float v = sm.st[0][u], g1 = sm.st[1][u], g2 = 0.0f, fr = 0.0f, in_e, in_i;
    if (MODEL != SZSNN_IZHIKEVICH) { g2 = sm.st[2][u]; fr = sm.st[3][u]; }
    if (FIXED) {
        in_e = __ll2float_rn(sm.fe[u]) * (1.0f / 4294967296.0f);
        in_i = __ll2float_rn(sm.fi[u]) * (1.0f / 4294967296.0f);
        sm.fe[u] = 0;
        sm.fi[u] = 0;
    } else {
        in_e = sm.ie[u];
        in_i = sm.ii[u];
        sm.ie[u] = 0.0f;
        sm.ii[u] = 0.0f;
    }
    const float i_ext = current ? current[id] : 0.0f;
    if (nd.dbg_in_e) { nd.dbg_in_e[id] = in_e; nd.dbg_in_i[id] = in_i; }
    const SharedParams sp{P.p};
    bool spk;
    if (MODEL == SZSNN_IF_CURR_EXP) spk = sz_if_curr_exp(sp, v, g1, g2, fr, in_e, in_i, i_ext, f, sp(12), sp(13));
    else if (MODEL == SZSNN_IF_COND_EXP) spk = sz_if_cond_exp(sp, v, g1, g2, fr, in_e, in_i, i_ext, f, sp(12), sp(13));
    else spk = sz_izhikevich(sp, v, g1, in_e, in_i, i_ext, f, (P.flags & SZSNN_POP_IZH_HALF_STEPS) != 0);
    sm.st[0][u] = v;
    sm.st[1][u] = g1;
    if (MODEL != SZSNN_IZHIKEVICH) { sm.st[2][u] = g2; sm.st[3][u] = fr; }
    return spk;
}

// The whole inline tile with population slot PI and model MODEL: bulk load,
// then the nd.upt sub-tiles, each ending in the spike epilogue.
template <int MODEL, bool FIXED, int PI>
__device__ __forceinline__ void tile_run(const NetDev& nd, const InBuf& inb, int64_t tile0, long long t,
                                        const uint32_t* __restrict__ forced, const float* __restrict__ current,
                                        uint32_t* __restrict__ out_words, unsigned char* smem, int phase)
{
    const uint32_t bs = blockDim.x, T = (uint32_t)nd.upt * bs, lane = threadIdx.x & 31;
    const TileSmem sm = tile_smem(smem, T, FIXED);
    const bool ok = tile_load<MODEL, FIXED>(nd, inb, tile0, T, sm, phase);
    const PopDev& P = nd.ipop[PI];
#pragma unroll 1
    for (int j = 0; j < nd.upt; ++j) {
        const uint32_t u = (uint32_t)j * bs + threadIdx.x;
        const int64_t id = tile0 + u;
        bool spk = false;
        if (ok && id < nd.U && owned(nd, id)) spk = tile_unit<MODEL, FIXED>(nd, P, inb, sm, (uint32_t)id, u, t, forced, current);
        __syncwarp();
        update_spikes(nd, t, id, spk, lane, out_words);
    }
    // the tile's new state and cleared inputs, back to global memory from
    // shared memory in one bulk store per array (units not updated here are
    // stored back as they were loaded)
    if (MODEL == SZSNN_POISSON) return;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the threads' writes, to the bulk copy engine
    if (!__syncthreads_and(ok ? 1 : 0)) return;  // a tile whose copies timed out is not stored (block-uniform)
    if (threadIdx.x == 0) {
        const int64_t n = min((int64_t)T, nd.U - tile0);
        const uint32_t b4 = (uint32_t)((n * 4 + 15) & ~(int64_t)15);
        const uint32_t b8 = (uint32_t)((n * 8 + 15) & ~(int64_t)15);
        const int nst = MODEL == SZSNN_IZHIKEVICH ? 2 : 4;
        float* const gst[4] = {nd.st0, nd.st1, nd.st2, nd.st3};
        for (int k = 0; k < nst; ++k) bulk_store(gst[k] + tile0, sm.st[k], b4);
        if (FIXED) {
            bulk_store(inb.fe + tile0, sm.fe, b8);
            bulk_store(inb.fi + tile0, sm.fi, b8);
        } else {
            bulk_store(inb.e + tile0, sm.ie, b4);
            bulk_store(inb.i + tile0, sm.ii, b4);
        }
        bulk_commit();
        bulk_wait_read();  // the sources are read before the block leaves or reloads its tile
    }
}

template <bool FIXED, int PI>
__device__ __forceinline__ void tile_run_pop(const NetDev& nd, const InBuf& inb, int64_t tile0, long long t,
                                            const uint32_t* __restrict__ forced, const float* __restrict__ current,
                                            uint32_t* __restrict__ out_words, unsigned char* smem, int phase)
{
    switch (nd.ipop[PI].model) {
    case SZSNN_IF_CURR_EXP: tile_run<SZSNN_IF_CURR_EXP, FIXED, PI>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    case SZSNN_IF_COND_EXP: tile_run<SZSNN_IF_COND_EXP, FIXED, PI>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    case SZSNN_IZHIKEVICH: tile_run<SZSNN_IZHIKEVICH, FIXED, PI>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    default: tile_run<SZSNN_POISSON, FIXED, PI>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    }
}

template <bool FIXED>
__device__ __forceinline__ void tile_run_slot(const NetDev& nd, int slot, const InBuf& inb, int64_t tile0, long long t,
                                             const uint32_t* __restrict__ forced, const float* __restrict__ current,
                                             uint32_t* __restrict__ out_words, unsigned char* smem, int phase)
{
    static_assert(INLINE_POPS == 4, "one case per parameter-table slot");
    switch (slot) {
    case 0: tile_run_pop<FIXED, 0>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    case 1: tile_run_pop<FIXED, 1>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    case 2: tile_run_pop<FIXED, 2>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    default: tile_run_pop<FIXED, 3>(nd, inb, tile0, t, forced, current, out_words, smem, phase); break;
    }
}

// Generic update: the block stages the populations overlapping its tile in
// shared memory once, then each thread finds the population of each of its
// units.  Handles per-unit parameters, Const_rate sources, tiles spanning
// populations and population tables larger than the parameter table.
struct StagedPops {
    const PopDev* pop;  // shared-memory copy
    int np;             // populations staged, -1 when more overlap the tile (global lookup)
};

__device__ __forceinline__ StagedPops stage_pops(const NetDev& nd, int blk)
{
    __shared__ PopDev s_pop[UPD_BLOCK_POPS];
    __shared__ int s_np;
    // populations overlapping the tile: the whole table when it is small, else
    // the host-computed (first, count) of this tile; one cooperative copy
    int first = 0, np = nd.npops;
    if (np > UPD_BLOCK_POPS) {
        const int2 fc = nd.blk_pop[blk];
        first = fc.x;
        np = fc.y > UPD_BLOCK_POPS ? -1 : fc.y;
    }
    if (np > 0) {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(nd.pops + first);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(s_pop);
        for (int w = threadIdx.x; w < np * (int)(sizeof(PopDev) / 8); w += blockDim.x) dst[w] = src[w];
    }
    if (threadIdx.x == 0) s_np = np;
    __syncthreads();
    return StagedPops{s_pop, s_np};
}

__device__ __forceinline__ bool update_generic(const NetDev& nd, const StagedPops& sp_, int64_t id, const InBuf& inb,
                                               long long t, UnitIn& a)
{
    const bool unit = id < nd.U && owned(nd, id), neuron = id < nd.N;
    const PopDev* pd = nullptr;
    if (unit) {
        if (sp_.np >= 0) {
            for (int i = 0; i < sp_.np; ++i)
                if (id >= sp_.pop[i].begin && id < sp_.pop[i].end) { pd = &sp_.pop[i]; break; }
        } else {
            const int pi = find_pop(nd.pops, nd.npops, id);
            if (pi >= 0 && id < nd.pops[pi].end) pd = &nd.pops[pi];
        }
    }
    bool spk = false;
    if (pd) {
        const int model = pd->model;
        if (neuron) {
            if (nd.acc_mode == SZSNN_ACC_FIXED) {
                a.in_e = __ll2float_rn(a.fxe) * (1.0f / 4294967296.0f);
                a.in_i = __ll2float_rn(a.fxi) * (1.0f / 4294967296.0f);
                inb.fe[id] = 0;
                inb.fi[id] = 0;
            } else {
                inb.e[id] = 0.0f;
                inb.i[id] = 0.0f;
            }
            if (nd.dbg_in_e) { nd.dbg_in_e[id] = a.in_e; nd.dbg_in_i[id] = a.in_i; }
            if (pd->pn) spk = run_neuron(UnitParams{pd->pn, id - pd->begin, pd->end - pd->begin}, model, pd->flags,
                                         a.v, a.g1, a.g2, a.fr, a.in_e, a.in_i, a.i_ext, a.f);
            else spk = run_neuron(SharedParams{pd->p}, model, pd->flags, a.v, a.g1, a.g2, a.fr, a.in_e, a.in_i,
                                  a.i_ext, a.f);
            nd.st0[id] = a.v;
            nd.st1[id] = a.g1;
            if (model != SZSNN_IZHIKEVICH) { nd.st2[id] = a.g2; nd.st3[id] = a.fr; }
        } else if (model == SZSNN_POISSON) {
            const float prob = pd->pn ? pd->pn[id - pd->begin] : pd->p[0];
            spk = sz_poisson_fires(pd->seed, id - pd->begin, t, prob) || a.f;
        } else if (model == SZSNN_CONST_RATE) {
            if (pd->pn) spk = sz_const_rate(UnitParams{pd->pn, id - pd->begin, pd->end - pd->begin}, a.v, a.f);
            else spk = sz_const_rate(SharedParams{pd->p}, a.v, a.f);
            nd.st0[id] = a.v;
        }
    }
    return spk;
}

// The loads of one unit (state, the inputs of step t from the parity buffer
// the host names, forced spike, external current).
__device__ __forceinline__ void load_unit(const NetDev& nd, const InBuf& inb, int64_t id,
                                          const uint32_t* __restrict__ forced, const float* __restrict__ current,
                                          UnitIn& a)
{
    a = UnitIn{};
    if (id >= nd.U) return;
    const uint32_t u = (uint32_t)id;
    a.v = nd.st0[u];
    if (id < nd.N) {
        a.g1 = nd.st1[u];
        a.g2 = nd.st2[u];
        a.fr = nd.st3[u];
        if (nd.acc_mode == SZSNN_ACC_FIXED) { a.fxe = inb.fe[u]; a.fxi = inb.fi[u]; }
        else { a.in_e = inb.e[u]; a.in_i = inb.i[u]; }
        if (current) a.i_ext = current[u];
    }
    if (forced) a.f = ((forced[u >> 5] >> (u & 31)) & 1u) != 0u;
}

// Block b covers units [b * T, (b + 1) * T), T = nd.upt * blockDim.x.  A
// block the host marked as lying inside one population of the parameter
// table runs an inline tile; other blocks run the generic update one
// block-size sub-tile at a time (thread's unit j * blockDim.x + threadIdx.x),
// each sub-tile ending in the spike epilogue, so every warp's units of a
// sub-tile are 32 consecutive ids (one raster word).
// Overlapped stepping: the warps with spikes deliver their units' m = 1
// buckets into the buffer of t+1, and block 0 does the per-step bookkeeping.
// phase: -1 for a block with one tile, else the persistent block's count of
// loaded tiles so far.  Returns whether this tile used the mbarrier.
__device__ __forceinline__ bool update_body(const NetDev& nd, int k_off, int blk, const uint32_t* __restrict__ forced,
                                            const float* __restrict__ current, uint32_t* __restrict__ out_words,
                                            int phase = -1)
{
    extern __shared__ __align__(128) unsigned char upd_smem[];
    const uint32_t bs = blockDim.x;
    const int64_t tile0 = (int64_t)blk * nd.upt * bs;
    const uint32_t lane = threadIdx.x & 31;
    const long long t = *nd.clock + k_off;
    const InBuf inb = in_buf_k(nd, k_off);
    int slot = -1;
#pragma unroll
    for (int i = 0; i < INLINE_POPS; ++i)
        if (blk >= nd.ib_lo[i] && blk < nd.ib_hi[i]) slot = i;
    bool used = false;
    if (slot >= 0) {
        if (nd.acc_mode == SZSNN_ACC_FIXED) tile_run_slot<true>(nd, slot, inb, tile0, t, forced, current, out_words, upd_smem, phase);
        else tile_run_slot<false>(nd, slot, inb, tile0, t, forced, current, out_words, upd_smem, phase);
        used = nd.ipop[slot].model != SZSNN_POISSON;
    } else {
        const StagedPops sp_ = stage_pops(nd, blk);
#pragma unroll 1
        for (int j = 0; j < nd.upt; ++j) {
            const int64_t id = tile0 + (int64_t)j * bs + threadIdx.x;
            UnitIn a;
            load_unit(nd, inb, id, forced, current, a);
            const bool spk = update_generic(nd, sp_, id, inb, t, a);
            __syncwarp();
            update_spikes(nd, t, id, spk, lane, out_words);
        }
    }
    if (nd.overlap && blk == 0 && threadIdx.x == 0) {
        step_bookkeeping(nd, t);
        // the inputs were read by the launch's parity, the deliveries write by
        // the step counter's: they must name the same buffer
        if (((uint64_t)t ^ (uint64_t)(nd.par0 + (uint32_t)k_off)) & 1u)
            dev_error(nd.err, SZSNN_DEV_STEP_PARITY, (uint32_t)t);
    }
    return used;
}

// ---- persistent warp tiles
//
// Each warp of the update grid streams warp tiles of WT = 128 consecutive
// units (four raster words: lane l handles units 32 j + l, j = 0..3) through
// a two-stage ring in its own slice of shared memory: while it updates tile
// k from one stage, the bulk copies of its next tile (k + number of update
// warps) fill the other.  A tile lying inside one population of the
// parameter table is updated in place in shared memory and written back
// with bulk stores (state and the cleared inputs); other tiles (population
// boundaries) run the generic per-unit update from global memory.  No block
// barrier is involved: a warp that waits on its spikes' delay-1 deliveries
// holds up only itself, and the warps of a block drift apart freely.
// Dynamic shared memory per warp: wt_region_bytes (two stages, two mbarriers).
#define WT 128
__host__ __device__ __forceinline__ constexpr uint32_t wt_stage_bytes(bool fixed) { return WT * (16u + (fixed ? 16u : 8u)); }
__host__ __device__ __forceinline__ size_t wt_region_bytes(bool fixed) { return 2 * (size_t)wt_stage_bytes(fixed) + 16; }

// arrays of a stage: st0..st3 (WT floats each), then the exc / inh inputs
// (WT floats or WT int64 each)
__device__ __forceinline__ float* wt_st(unsigned char* stage, int k) { return reinterpret_cast<float*>(stage) + k * WT; }
__device__ __forceinline__ float* wt_ie(unsigned char* stage) { return reinterpret_cast<float*>(stage) + 4 * WT; }
__device__ __forceinline__ float* wt_ii(unsigned char* stage) { return reinterpret_cast<float*>(stage) + 5 * WT; }
__device__ __forceinline__ long long* wt_fe(unsigned char* stage) { return reinterpret_cast<long long*>(stage + 16 * WT); }
__device__ __forceinline__ long long* wt_fi(unsigned char* stage) { return reinterpret_cast<long long*>(stage + 24 * WT); }

// slot of the parameter table whose population holds units [u0, u0 + WT) of
// the network, or -1
__device__ __forceinline__ int wt_slot(const NetDev& nd, int64_t u0)
{
    const int64_t u1 = min(u0 + (int64_t)WT, nd.U);
#pragma unroll
    for (int i = 0; i < INLINE_POPS; ++i)
        if (nd.ipop[i].end > nd.ipop[i].begin && u0 >= nd.ipop[i].begin && u1 <= nd.ipop[i].end) return i;
    return -1;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (int i = 0; i < (1 << 20); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// bulk copies of the tile at u0 (model MODEL) into a stage, completing on bar
// (one thread); Poisson tiles read nothing
template <int MODEL, bool FIXED>
__device__ __forceinline__ void wt_issue(const NetDev& nd, const InBuf& inb, int64_t u0, unsigned char* sm,
                                         uint64_t* bar)
{
    if (MODEL == SZSNN_POISSON) return;
    const int64_t n = min((int64_t)WT, nd.U - u0);
    const uint32_t b4 = (uint32_t)((n * 4 + 15) & ~(int64_t)15);
    const uint32_t b8 = (uint32_t)((n * 8 + 15) & ~(int64_t)15);
    const int nst = MODEL == SZSNN_IZHIKEVICH ? 2 : 4;
    const uint32_t total = (uint32_t)nst * b4 + 2u * (FIXED ? b8 : b4);
    asm volatile("{\n .reg .b64 s;\n mbarrier.arrive.expect_tx.shared::cta.b64 s, [%0], %1;\n}"
                 :: "r"(smem_addr(bar)), "r"(total) : "memory");
    float* const gst[4] = {nd.st0, nd.st1, nd.st2, nd.st3};
    for (int k = 0; k < nst; ++k) bulk_load(wt_st(sm, k), gst[k] + u0, b4, bar);
    if (FIXED) {
        bulk_load(wt_fe(sm), inb.fe + u0, b8, bar);
        bulk_load(wt_fi(sm), inb.fi + u0, b8, bar);
    } else {
        bulk_load(wt_ie(sm), inb.e + u0, b4, bar);
        bulk_load(wt_ii(sm), inb.i + u0, b4, bar);
    }
}

// issue for the tile at u0 in slot `slot` (>= 0); returns whether copies were issued
template <bool FIXED>
__device__ __forceinline__ bool wt_issue_slot(const NetDev& nd, int slot, const InBuf& inb, int64_t u0,
                                              unsigned char* sm, uint64_t* bar)
{
    switch (nd.ipop[slot].model) {
    case SZSNN_IF_CURR_EXP: wt_issue<SZSNN_IF_CURR_EXP, FIXED>(nd, inb, u0, sm, bar); return true;
    case SZSNN_IF_COND_EXP: wt_issue<SZSNN_IF_COND_EXP, FIXED>(nd, inb, u0, sm, bar); return true;
    case SZSNN_IZHIKEVICH: wt_issue<SZSNN_IZHIKEVICH, FIXED>(nd, inb, u0, sm, bar); return true;
    default: return false;
    }
}

// Update the tile at u0 in place in its stage (slot PI, model MODEL), each
// 32-unit sub-tile ending in the spike epilogue; then the stage's state and
// cleared inputs go back to global memory by bulk stores issued by lane 0.
template <int MODEL, bool FIXED, int PI>
__device__ __forceinline__ void wt_run(const NetDev& nd, const InBuf& inb, unsigned char* sm, int64_t u0, long long t,
                                       bool ok, const uint32_t* __restrict__ forced,
                                       const float* __restrict__ current, uint32_t* __restrict__ out_words)
{
    const uint32_t lane = threadIdx.x & 31;
    const PopDev& P = nd.ipop[PI];
    const SharedParams sp{P.p};
#pragma unroll 1
    for (int j = 0; j < WT / 32; ++j) {
        const uint32_t u = 32u * j + lane;
        const int64_t id = u0 + u;
        bool spk = false;
        if (ok && id < nd.U && owned(nd, id)) {
            const bool f = forced ? ((forced[id >> 5] >> (id & 31)) & 1u) != 0u : false;
            if (MODEL == SZSNN_POISSON) {
                spk = sz_poisson_fires(P.seed, id - P.begin, t, P.p[0]) || f;
            } else {
                float v = wt_st(sm, 0)[u], g1 = wt_st(sm, 1)[u], g2 = 0.0f, fr = 0.0f, in_e, in_i;
                if (MODEL != SZSNN_IZHIKEVICH) { g2 = wt_st(sm, 2)[u]; fr = wt_st(sm, 3)[u]; }
                if (FIXED) {
                    in_e = __ll2float_rn(wt_fe(sm)[u]) * (1.0f / 4294967296.0f);
                    in_i = __ll2float_rn(wt_fi(sm)[u]) * (1.0f / 4294967296.0f);
                    wt_fe(sm)[u] = 0;
                    wt_fi(sm)[u] = 0;
                } else {
                    in_e = wt_ie(sm)[u];
                    in_i = wt_ii(sm)[u];
                    wt_ie(sm)[u] = 0.0f;
                    wt_ii(sm)[u] = 0.0f;
                }
                const float i_ext = current ? current[id] : 0.0f;
                if (nd.dbg_in_e) { nd.dbg_in_e[id] = in_e; nd.dbg_in_i[id] = in_i; }
                if (MODEL == SZSNN_IF_CURR_EXP) spk = sz_if_curr_exp(sp, v, g1, g2, fr, in_e, in_i, i_ext, f, sp(12), sp(13));
                else if (MODEL == SZSNN_IF_COND_EXP) spk = sz_if_cond_exp(sp, v, g1, g2, fr, in_e, in_i, i_ext, f, sp(12), sp(13));
                else spk = sz_izhikevich(sp, v, g1, in_e, in_i, i_ext, f, (P.flags & SZSNN_POP_IZH_HALF_STEPS) != 0);
                wt_st(sm, 0)[u] = v;
                wt_st(sm, 1)[u] = g1;
                if (MODEL != SZSNN_IZHIKEVICH) { wt_st(sm, 2)[u] = g2; wt_st(sm, 3)[u] = fr; }
            }
        }
        __syncwarp();
        update_spikes(nd, t, id, spk, lane, out_words);
    }
    if (MODEL == SZSNN_POISSON || !ok) return;
    // the lanes' shared-memory writes become visible to the bulk copy engine
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) {
        const int64_t n = min((int64_t)WT, nd.U - u0);
        const uint32_t b4 = (uint32_t)((n * 4 + 15) & ~(int64_t)15);
        const uint32_t b8 = (uint32_t)((n * 8 + 15) & ~(int64_t)15);
        const int nst = MODEL == SZSNN_IZHIKEVICH ? 2 : 4;
        float* const gst[4] = {nd.st0, nd.st1, nd.st2, nd.st3};
        for (int k = 0; k < nst; ++k) bulk_store(gst[k] + u0, wt_st(sm, k), b4);
        if (FIXED) {
            bulk_store(inb.fe + u0, wt_fe(sm), b8);
            bulk_store(inb.fi + u0, wt_fi(sm), b8);
        } else {
            bulk_store(inb.e + u0, wt_ie(sm), b4);
            bulk_store(inb.i + u0, wt_ii(sm), b4);
        }
        bulk_commit();
    }
}

template <bool FIXED, int PI>
__device__ __forceinline__ void wt_run_pop(const NetDev& nd, const InBuf& inb, unsigned char* sm, int64_t u0, long long t,
                                           bool ok, const uint32_t* __restrict__ forced,
                                           const float* __restrict__ current, uint32_t* __restrict__ out_words)
{
    switch (nd.ipop[PI].model) {
    case SZSNN_IF_CURR_EXP: wt_run<SZSNN_IF_CURR_EXP, FIXED, PI>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    case SZSNN_IF_COND_EXP: wt_run<SZSNN_IF_COND_EXP, FIXED, PI>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    case SZSNN_IZHIKEVICH: wt_run<SZSNN_IZHIKEVICH, FIXED, PI>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    default: wt_run<SZSNN_POISSON, FIXED, PI>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    }
}

template <bool FIXED>
__device__ __forceinline__ void wt_run_slot(const NetDev& nd, int slot, const InBuf& inb, unsigned char* sm, int64_t u0,
                                            long long t, bool ok, const uint32_t* __restrict__ forced,
                                            const float* __restrict__ current, uint32_t* __restrict__ out_words)
{
    static_assert(INLINE_POPS == 4, "one case per parameter-table slot");
    switch (slot) {
    case 0: wt_run_pop<FIXED, 0>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    case 1: wt_run_pop<FIXED, 1>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    case 2: wt_run_pop<FIXED, 2>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    default: wt_run_pop<FIXED, 3>(nd, inb, sm, u0, t, ok, forced, current, out_words); break;
    }
}

// The persistent update of one warp: warp gw of nw update warps takes warp
// tiles gw, gw + nw, ... (see the section comment).  Every bulk copy issued
// is waited for (bounded; device error 7 when a wait runs out, after which
// the warp stops taking tiles), and lane 0 waits for its bulk stores to have
// read their sources before the warp leaves.
template <bool FIXED>
__device__ __forceinline__ void update_warp_tiles(const NetDev& nd, int k_off, int gw, int nw,
                                                  const uint32_t* __restrict__ forced,
                                                  const float* __restrict__ current, uint32_t* __restrict__ out_words)
{
    extern __shared__ __align__(128) unsigned char upd_smem[];
    const uint32_t lane = threadIdx.x & 31;
    unsigned char* reg = upd_smem + (size_t)(threadIdx.x >> 5) * wt_region_bytes(FIXED);
    uint64_t* bar = reinterpret_cast<uint64_t*>(reg + 2 * wt_stage_bytes(FIXED));
    constexpr uint32_t SB = wt_stage_bytes(FIXED);
    const long long t = *nd.clock + k_off;
    const InBuf inb = in_buf_k(nd, k_off);
    const int nwt = (int)((nd.U + WT - 1) / WT);  // units < 2^31
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t ph = 0;        // bit s: parity of the next wait on stage s
    uint32_t pending = 0;   // lane 0: bit s set while stage s has copies not yet waited for
    if (lane == 0 && gw < nwt) {
        const int sl = wt_slot(nd, (int64_t)gw * WT);
        if (sl >= 0 && wt_issue_slot<FIXED>(nd, sl, inb, (int64_t)gw * WT, reg, &bar[0])) pending |= 1u;
    }
    int k = 0;
    for (int wt = gw; wt < nwt; wt += nw, ++k) {
        const int s = k & 1;
        const int nxt = wt + nw;
        if (lane == 0) {
            bulk_wait_read();  // the stores of the previous tile (stage s ^ 1) have read their sources
            if (nxt < nwt) {
                const int sl = wt_slot(nd, (int64_t)nxt * WT);
                if (sl >= 0 && wt_issue_slot<FIXED>(nd, sl, inb, (int64_t)nxt * WT, reg + (s ^ 1) * SB, &bar[s ^ 1]))
                    pending |= 1u << (s ^ 1);
            }
        }
        const int64_t u0 = (int64_t)wt * WT;
        const int slot = wt_slot(nd, u0);
        if (slot >= 0) {
            bool ok = true;
            if (nd.ipop[slot].model != SZSNN_POISSON) {
                ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bar[s], (ph >> s) & 1u));
                if (!ok) {  // report, wait once more so no copy is still writing the stage, stop
                    if (lane == 0) dev_error(nd.err, SZSNN_DEV_WAIT_TIMEOUT, (uint32_t)u0);
                    mbar_wait_bounded(&bar[s], (ph >> s) & 1u);
                }
                ph ^= 1u << s;
                pending &= ~(1u << s);
            }
            wt_run_slot<FIXED>(nd, slot, inb, reg + s * SB, u0, t, ok, forced, current, out_words);
            if (!ok) break;
        } else {
            const StagedPops gp{nd.pops, nd.npops};
#pragma unroll 1
            for (int j = 0; j < WT / 32; ++j) {
                const int64_t id = u0 + 32 * j + lane;
                UnitIn a;
                load_unit(nd, inb, id, forced, current, a);
                const bool spk = update_generic(nd, gp, id, inb, t, a);
                __syncwarp();
                update_spikes(nd, t, id, spk, lane, out_words);
            }
        }
    }
    if (lane == 0) {
        for (int s = 0; s < 2; ++s)  // copies issued for a tile the loop did not reach
            if (pending & (1u << s)) mbar_wait_bounded(&bar[s], (ph >> s) & 1u);
        bulk_wait_read();
    }
    __syncwarp();
    if (nd.overlap && gw == 0 && lane == 0) {
        step_bookkeeping(nd, t);
        if (((uint64_t)t ^ (uint64_t)(nd.par0 + (uint32_t)k_off)) & 1u)
            dev_error(nd.err, SZSNN_DEV_STEP_PARITY, (uint32_t)t);
    }
}

// Persistent block tiles: update block blk of nblk takes tiles blk, blk +
// nblk, ... of the block-tile scheme, one after the other, with one
// mbarrier (initialised once) whose phase per loaded tile the block counts;
// a block barrier separates the tiles (shared memory reused).  Blocks are
// launched once per step, as many as stay resident, so no block is
// scheduled mid-step and no partial wave trails the launch.
__device__ __forceinline__ void update_persistent(const NetDev& nd, int k_off, int blk, int nblk,
                                                  const uint32_t* __restrict__ forced,
                                                  const float* __restrict__ current, uint32_t* __restrict__ out_words)
{
    extern __shared__ __align__(128) unsigned char upd_smem[];
    const int64_t ntiles = sz_div_up(nd.U, (int64_t)nd.upt * blockDim.x);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(upd_smem)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __shared__ int s_stop;
    __syncthreads();
    int phase = 0;
    for (int64_t tile = blk; tile < ntiles; tile += nblk) {
        if (update_body(nd, k_off, (int)tile, forced, current, out_words, phase)) ++phase;
        // a bulk-copy wait that ran out (device error 7) ends the block's
        // tiles: a copy might still be in flight into its shared memory
        if (threadIdx.x == 0) s_stop = *reinterpret_cast<volatile uint32_t*>(nd.err) == SZSNN_DEV_WAIT_TIMEOUT;
        __syncthreads();  // every thread is done with the tile's shared memory
        if (s_stop) break;
    }
}

// update with one tile scheme (MODE 0: a block per tile, 1: persistent warp
// tiles, 2: persistent block tiles), for update block `blk` of `nblk`
template <int MODE>
__device__ __forceinline__ void update_any(const NetDev& nd, int k_off, int blk, int nblk,
                                           const uint32_t* __restrict__ forced, const float* __restrict__ current,
                                           uint32_t* __restrict__ out_words)
{
    if constexpr (MODE == 1) {
        const int wpb = (int)(blockDim.x >> 5);
        const int gw = blk * wpb + (int)(threadIdx.x >> 5), nw = nblk * wpb;
        if (nd.acc_mode == SZSNN_ACC_FIXED) update_warp_tiles<true>(nd, k_off, gw, nw, forced, current, out_words);
        else update_warp_tiles<false>(nd, k_off, gw, nw, forced, current, out_words);
    } else if constexpr (MODE == 2) {
        update_persistent(nd, k_off, blk, nblk, forced, current, out_words);
    } else {
        update_body(nd, k_off, blk, forced, current, out_words);
    }
}

// registers: block tiles keep six resident 256-thread blocks per SM (40
// registers); warp tiles are bound by their shared-memory ring to four
#define UPD_MIN_BLOCKS_WT 4

template <int MODE>
__global__ void __launch_bounds__(UPD_MAX_BLOCK, MODE == 1 ? UPD_MIN_BLOCKS_WT : UPD_MIN_BLOCKS)
    k_update(const __grid_constant__ NetDev nd, int k_off, const uint32_t* __restrict__ forced,
             const float* __restrict__ current, uint32_t* __restrict__ out_words)
{
    update_any<MODE>(nd, k_off, blockIdx.x, gridDim.x, forced, current, out_words);
}

// Overlapped step t in one launch: blocks 0..far_blocks-1 deliver delays >= 2
// into step t+1's inputs (reading ring slots <= t-1 only), the others update
// step t (which delivers its own spikes' delay-1 buckets into step t+1).  The
// delivery blocks come first so they are resident from the start and run
// beside the update blocks.
template <int G, int MODE>
__global__ void __launch_bounds__(UPD_MAX_BLOCK, MODE == 1 ? UPD_MIN_BLOCKS_WT : UPD_MIN_BLOCKS)
    k_step(const __grid_constant__ NetDev nd, int k_off, int far_blocks, const uint32_t* __restrict__ forced,
           const float* __restrict__ current, uint32_t* __restrict__ out_words)
{
    if ((int)blockIdx.x < far_blocks) {  // G > 0: grouped delivery, G lanes per bucket; G < 0: flattened, -G items per warp
        if constexpr (G > 0) propagate_grouped<G>(nd, k_off + 1, 2, PF_PENDING, blockIdx.x, far_blocks);
        else propagate_flat<-G>(nd, k_off + 1, 2, PF_PENDING, blockIdx.x, far_blocks);
        return;
    }
    update_any<MODE>(nd, k_off, blockIdx.x - far_blocks, gridDim.x - far_blocks, forced, current, out_words);
}

// Spikes of the step just done (step counter - 1) emitted by units another
// shard updates: one warp per 32-unit word, each set bit handled as the
// update's spike epilogue handles its own spikes (group counter, ring
// append to slot t, and in the overlapped order the delay-1 delivery into
// step t+1's inputs; the classic order delivers it from the ring).
__global__ void __launch_bounds__(256) k_inject(const __grid_constant__ NetDev nd, const uint32_t* __restrict__ words)
{
    const long long t = *nd.clock - 1;
    const uint32_t lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nd.words; w += nw) {
        const uint32_t word = words[w];
        if (!word) continue;  // warp-uniform
        const int64_t id = w * 32 + lane;
        const bool spk = ((word >> lane) & 1u) && id < nd.U;
        update_spikes(nd, t, id, spk, lane, nullptr);
    }
}

// ---- resident stepping
//
// One cooperative launch runs a whole chunk of overlapped steps with the
// neurons' state held in shared memory across the steps.  One block per SM,
// each owning a contiguous range of neuron words and one of source words
// (word-aligned, so every raster word has one writer).  Per step t the
// block's first `uw` warps update its units (inputs read through L2 and
// cleared, state from and to shared memory, the spike epilogue of the tile
// update: ring append, raster word, delay-1 delivery into step t+1); its
// other warps take their share of the far delivery into step t+1 (delays
// >= 2, ring slots <= t-1), split over the delivery warps of all blocks.  A
// bounded grid barrier ends the step: update(t+1) needs every delivery into
// step t+1 and every ring append of step t.  Per step a neuron moves only its
// inputs through L2 (read and clear), not its state.  Data written inside
// the launch (ring counts and ids, inputs, statistics) is read with L2 loads.
struct ResSync {
    unsigned int count;  // arrivals: one per block per step
    unsigned int abort;  // set by a block whose wait ran out
};

struct ResRange {
    int64_t n_lo, n_cnt;  // neuron words of the block, as unit ids (32 per word)
    int64_t s_lo, s_cnt;  // source words (those after the word holding the last neuron)
};

__host__ __device__ __forceinline__ ResRange res_range(int64_t N, int64_t words, int b, int nb)
{
    const int64_t nw = sz_div_up(N, 32), sw = words - nw;
    const int64_t a0 = nw * b / nb, a1 = nw * (b + 1) / nb;
    const int64_t c0 = nw + sw * b / nb, c1 = nw + sw * (b + 1) / nb;
    return ResRange{32 * a0, 32 * (a1 - a0), 32 * c0, 32 * (c1 - c0)};
}

// neuron slots of a block's shared state: its largest neuron range
__host__ __device__ __forceinline__ int64_t res_cap(int64_t N, int nb) { return 32 * sz_div_up(sz_div_up(N, 32), nb); }

#define RES_THREADS 1024
#define RES_UB 4                 // units per update thread in flight (loads issued together)
#define RES_WAIT_ITERS (1 << 21)  // grid-barrier polls before a block gives up (about a second)

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void named_sync(int id, int threads)
{
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(threads) : "memory");
}

// Bounded grid barrier.  Thread 0 first adds the block's delivered events of
// the step to the pending counter of step t+1, then arrives and polls; every
// write of the block before the barrier is visible to every block after it.
// Returns false when a wait ran out here or in another block (device error 7
// is recorded): the kernel then stops stepping.
__device__ __forceinline__ bool res_grid_sync(const NetDev& nd, ResSync* s, unsigned int target, int* s_flag,
                                              unsigned long long* s_ev, unsigned long long* pending)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        if (*s_ev) { atomicAdd(pending, *s_ev); *s_ev = 0; }
        __threadfence();
        atomicAdd(&s->count, 1u);
        int ok = 0;
        for (int i = 0; i < RES_WAIT_ITERS; ++i) {
            if (ld_acquire_u32(&s->count) >= target) { ok = 1; break; }
            if (*reinterpret_cast<volatile unsigned int*>(&s->abort)) break;
            if (i >= 16) __nanosleep(64);
        }
        if (!ok) {
            atomicExch(&s->abort, 1u);
            dev_error(nd.err, SZSNN_DEV_WAIT_TIMEOUT, target);
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// One population's parameters in registers (constant slot indices; the
// slots a model does not read are never loaded)
struct RegParams {
    float p[POP_SLOTS];
    __device__ __forceinline__ float operator()(int k) const { return p[k]; }
};

// A batch of RES_UB units per thread, all in population P of neuron model
// MODEL (warp-uniform): state loads from shared memory for every unit first,
// then the model arithmetic on registers (independent units, so their
// instruction chains interleave), then the stores.  Arithmetic as
// tile_unit's; act[u]: the unit is updated; id[u] - n_lo: its shared-memory
// slot.
template <int MODEL>
__device__ __forceinline__ void res_batch(const PopDev& P, float* const* st, const InBuf& inb, bool fixed,
                                          const uint32_t* id, uint32_t n_lo, const bool* act, const float* in_e,
                                          const float* in_i, const float* ext, const bool* f, bool* spk)
{
    RegParams rp;
#pragma unroll
    for (int k = 0; k < POP_SLOTS; ++k) rp.p[k] = P.p[k];
    const bool half = (P.flags & SZSNN_POP_IZH_HALF_STEPS) != 0;
    float v[RES_UB], g1[RES_UB], g2[RES_UB], fr[RES_UB];
#pragma unroll
    for (int u = 0; u < RES_UB; ++u) {
        v[u] = g1[u] = g2[u] = fr[u] = 0.0f;
        if (act[u]) {
            v[u] = st[0][(id[u] - n_lo)];
            g1[u] = st[1][(id[u] - n_lo)];
            if (MODEL != SZSNN_IZHIKEVICH) { g2[u] = st[2][(id[u] - n_lo)]; fr[u] = st[3][(id[u] - n_lo)]; }
        }
    }
#pragma unroll
    for (int u = 0; u < RES_UB; ++u) {
        bool s;
        if (MODEL == SZSNN_IF_CURR_EXP)
            s = sz_if_curr_exp(rp, v[u], g1[u], g2[u], fr[u], in_e[u], in_i[u], ext[u], f[u], rp(12), rp(13));
        else if (MODEL == SZSNN_IF_COND_EXP)
            s = sz_if_cond_exp(rp, v[u], g1[u], g2[u], fr[u], in_e[u], in_i[u], ext[u], f[u], rp(12), rp(13));
        else
            s = sz_izhikevich(rp, v[u], g1[u], in_e[u], in_i[u], ext[u], f[u], half);
        spk[u] = act[u] && s;
    }
#pragma unroll
    for (int u = 0; u < RES_UB; ++u) {
        if (!act[u]) continue;
        st[0][(id[u] - n_lo)] = v[u];
        st[1][(id[u] - n_lo)] = g1[u];
        if (MODEL != SZSNN_IZHIKEVICH) { st[2][(id[u] - n_lo)] = g2[u]; st[3][(id[u] - n_lo)] = fr[u]; }
        if (fixed) { inb.fe[id[u]] = 0; inb.fi[id[u]] = 0; }
        else { inb.e[id[u]] = 0.0f; inb.i[id[u]] = 0.0f; }
    }
}

// The update warps' units of step t: the block's neuron ids, then its source
// ids, RES_UB per thread at a time (the batch's loads in flight together);
// warp w's lanes hold 32 consecutive ids, one raster word.  A batch whose
// active units all lie in one population (warp-uniform) runs that model's
// batch update; others run unit by unit.  Arithmetic and side effects as the
// generic update's (update_generic), with the state in shared memory slot
// id - n_lo.  Ids fit 32 bits (resident networks hold a few million units).
template <bool FIXED>
__device__ __forceinline__ void res_update(const NetDev& nd, const PopDev* __restrict__ sp, const ResRange& rr,
                                           float* const* st, long long t, const uint32_t* __restrict__ forced,
                                           const float* __restrict__ current, uint32_t* __restrict__ out_words,
                                           int nthr, bool all_owned)
{
    const InBuf inb = in_buf(nd, t);
    const uint32_t lane = threadIdx.x & 31, wbase = threadIdx.x & ~31u;
    const uint32_t n_lo = (uint32_t)rr.n_lo, n_cnt = (uint32_t)rr.n_cnt, s_lo = (uint32_t)rr.s_lo;
    const uint32_t total = (uint32_t)(rr.n_cnt + rr.s_cnt);  // a multiple of 32
    const uint32_t N = (uint32_t)nd.N, U = (uint32_t)nd.U;
    const int np = nd.npops;
    for (uint32_t i0 = 0; i0 < total; i0 += (uint32_t)nthr * RES_UB) {
        uint32_t id[RES_UB];
        float in_e[RES_UB], in_i[RES_UB], ext[RES_UB];
        bool f[RES_UB], act[RES_UB], spk[RES_UB];
        int pi[RES_UB];
#pragma unroll
        for (int u = 0; u < RES_UB; ++u) {
            const uint32_t i = i0 + (uint32_t)u * nthr + threadIdx.x;
            id[u] = i < n_cnt ? n_lo + i : s_lo + (i - n_cnt);
            in_e[u] = in_i[u] = ext[u] = 0.0f;
            f[u] = false;
            act[u] = i < total && id[u] < U && (all_owned || owned(nd, id[u]));
            pi[u] = -1;
            if (!act[u]) continue;
            for (int k = 0; k < np; ++k)
                if (id[u] >= sp[k].begin && id[u] < sp[k].end) pi[u] = k;
            if (pi[u] < 0) act[u] = false;
            if (act[u] && id[u] < N) {
                if (FIXED) {
                    in_e[u] = __ll2float_rn(__ldcg(&inb.fe[id[u]])) * (1.0f / 4294967296.0f);
                    in_i[u] = __ll2float_rn(__ldcg(&inb.fi[id[u]])) * (1.0f / 4294967296.0f);
                } else {
                    in_e[u] = __ldcg(&inb.e[id[u]]);
                    in_i[u] = __ldcg(&inb.i[id[u]]);
                }
                if (current) ext[u] = current[id[u]];
            }
            if (forced && act[u]) f[u] = ((forced[id[u] >> 5] >> (id[u] & 31)) & 1u) != 0u;
        }
        // the batch's population when every active unit of the warp lies in one
        int mine = -2;
        bool uni = true;
#pragma unroll
        for (int u = 0; u < RES_UB; ++u)
            if (act[u]) {
                if (mine == -2) mine = pi[u];
                else if (pi[u] != mine) uni = false;
            }
        const int p0 = __reduce_max_sync(0xffffffffu, mine);
        uni = __all_sync(0xffffffffu, uni && (mine == -2 || mine == p0)) && p0 >= 0;
        if (uni && sp[p0].pn) uni = false;  // per-unit parameter tables: unit by unit
        if (uni) {
            const PopDev& P = sp[p0];
            if (P.model == SZSNN_IF_COND_EXP)
                res_batch<SZSNN_IF_COND_EXP>(P, st, inb, FIXED, id, n_lo, act, in_e, in_i, ext, f, spk);
            else if (P.model == SZSNN_IF_CURR_EXP)
                res_batch<SZSNN_IF_CURR_EXP>(P, st, inb, FIXED, id, n_lo, act, in_e, in_i, ext, f, spk);
            else if (P.model == SZSNN_IZHIKEVICH)
                res_batch<SZSNN_IZHIKEVICH>(P, st, inb, FIXED, id, n_lo, act, in_e, in_i, ext, f, spk);
            else {
#pragma unroll
                for (int u = 0; u < RES_UB; ++u)
                    spk[u] = act[u] && (sz_poisson_fires(P.seed, (int64_t)id[u] - P.begin, t, P.p[0]) || f[u]);
            }
        } else {
#pragma unroll
            for (int u = 0; u < RES_UB; ++u) {
                spk[u] = false;
                if (!act[u]) continue;
                const PopDev& P = sp[pi[u]];
                if (id[u] < N) {
                    float v = st[0][(id[u] - n_lo)], g1 = st[1][(id[u] - n_lo)], g2 = 0.0f, fr = 0.0f;
                    if (P.model != SZSNN_IZHIKEVICH) { g2 = st[2][(id[u] - n_lo)]; fr = st[3][(id[u] - n_lo)]; }
                    if (P.pn)
                        spk[u] = run_neuron(UnitParams{P.pn, (int64_t)id[u] - P.begin, P.end - P.begin}, P.model,
                                            P.flags, v, g1, g2, fr, in_e[u], in_i[u], ext[u], f[u]);
                    else
                        spk[u] = run_neuron(SharedParams{P.p}, P.model, P.flags, v, g1, g2, fr, in_e[u], in_i[u],
                                            ext[u], f[u]);
                    st[0][(id[u] - n_lo)] = v;
                    st[1][(id[u] - n_lo)] = g1;
                    if (P.model != SZSNN_IZHIKEVICH) { st[2][(id[u] - n_lo)] = g2; st[3][(id[u] - n_lo)] = fr; }
                    if (FIXED) { inb.fe[id[u]] = 0; inb.fi[id[u]] = 0; }
                    else { inb.e[id[u]] = 0.0f; inb.i[id[u]] = 0.0f; }
                } else if (P.model == SZSNN_POISSON) {
                    const float prob = P.pn ? P.pn[(int64_t)id[u] - P.begin] : P.p[0];
                    spk[u] = sz_poisson_fires(P.seed, (int64_t)id[u] - P.begin, t, prob) || f[u];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < RES_UB; ++u) {
            if (i0 + (uint32_t)u * nthr + wbase >= total) continue;  // warp-uniform
            __syncwarp();
            update_spikes(nd, t, id[u], spk[u], lane, out_words);
        }
    }
}

// The delivery warps' share of the far delivery into step tt (delays 2..D):
// the ring counts scanned once per block (named barrier 1 over the delivery
// threads), then the flattened walk with L2 loads of the ring ids.
template <int IPW>
__device__ __forceinline__ void res_deliver(const NetDev& nd, long long tt, int64_t gw, int64_t nw, int dtid,
                                            int dthr, uint32_t* s_pre, int2* win, unsigned long long* s_ev,
                                            bool book)
{
    const int D = nd.D, R = D + 1;
    if (book && dtid == 0) step_bookkeeping(nd, tt - 1);  // its loads overlap the ring-count loads
    for (int m = dtid + 1; m <= D; m += dthr) {
        const long long tm = tt - m;
        s_pre[m] = (m >= 2 && tm >= 0) ? __ldcg(&nd.ring_cnt[tm % R]) : 0u;
    }
    if (dtid == 0) s_pre[0] = 0;
    named_sync(1, dthr);
    if (dtid < 32) {  // inclusive scan of counts over m = 1..D
        uint32_t carry = 0;
        const uint32_t lane = (uint32_t)dtid;
        for (int m0 = 1; m0 <= D; m0 += 32) {
            const int m = m0 + (int)lane;
            const uint32_t c = (m <= D) ? s_pre[m] : 0u;
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += y;
            }
            if (m <= D) s_pre[m] = carry + incl;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    named_sync(1, dthr);
    uint32_t ev = flat_items<IPW, true>(nd, tt, s_pre, gw, nw, win, in_buf(nd, tt));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ev += __shfl_down_sync(0xffffffffu, ev, o);
    if ((dtid & 31) == 0 && ev) atomicAdd(s_ev, (unsigned long long)ev);
}

// `len` overlapped steps from the step counter on; uw update warps per
// block, nst state slots kept (2: Izhikevich only, 4 otherwise); per-step
// forced words / currents / raster words at step k of the chunk arrays.
// Dynamic shared memory: the delivery warps' copy windows, then nst arrays of
// res_cap(N, gridDim.x) floats.
template <bool FIXED, int IPW>
__global__ void __launch_bounds__(RES_THREADS, 1)
    k_resident(const __grid_constant__ NetDev nd, ResSync* sync, long long* clock, int len, int uw, int nst,
               const uint32_t* __restrict__ forced, const float* __restrict__ current, uint32_t* __restrict__ raster)
{
    extern __shared__ __align__(128) unsigned char upd_smem[];
    __shared__ uint32_t s_pre[1025];
    __shared__ unsigned long long s_ev;
    __shared__ PopDev s_pop[INLINE_POPS];
    __shared__ int s_flag;
    const int b = blockIdx.x, nb = gridDim.x;
    const ResRange rr = res_range(nd.N, nd.words, b, nb);
    const int64_t cap = res_cap(nd.N, nb);
    const int warp = (int)(threadIdx.x >> 5), ndw = (int)(blockDim.x >> 5) - uw;
    int2* const win = reinterpret_cast<int2*>(upd_smem);
    float* const sb = reinterpret_cast<float*>(upd_smem + (size_t)ndw * 32 * FAR_WPL * sizeof(int2));
    float* const st[4] = {sb, sb + cap, nst > 2 ? sb + 2 * cap : nullptr, nst > 2 ? sb + 3 * cap : nullptr};
    float* const gst[4] = {nd.st0, nd.st1, nd.st2, nd.st3};
    if ((int)threadIdx.x < nd.npops) s_pop[threadIdx.x] = nd.pops[threadIdx.x];
    if (threadIdx.x == 0) s_ev = 0;
    for (int64_t i = threadIdx.x; i < rr.n_cnt; i += blockDim.x) {
        const int64_t id = rr.n_lo + i;
        if (id < nd.N) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < nst) st[k][i] = gst[k][id];
        }
    }
    const long long t0 = *clock;  // every block reads it before its first arrival; block 0 advances it after the last
    const bool all_owned = nd.own_lo[0] == 0 && nd.own_hi[0] == nd.N && nd.own_lo[1] == nd.N && nd.own_hi[1] == nd.U;
    __syncthreads();
    for (int k = 0; k < len; ++k) {
        const long long t = t0 + k;
        if (warp < uw) {
            if (b == 0 && threadIdx.x == 0 && nd.D < 2) step_bookkeeping(nd, t);
            res_update<FIXED>(nd, s_pop, rr, st, t, forced ? forced + (size_t)k * nd.words : nullptr,
                              current ? current + (size_t)k * (size_t)nd.N : nullptr,
                              raster ? raster + (size_t)k * nd.words : nullptr, uw * 32, all_owned);
        } else if (nd.D >= 2) {
            res_deliver<IPW>(nd, t + 1, (int64_t)b * ndw + (warp - uw), (int64_t)nb * ndw,
                             (int)threadIdx.x - uw * 32, ndw * 32, s_pre, win + (size_t)(warp - uw) * 32 * FAR_WPL,
                             &s_ev, b == 0);
        }
        if (!res_grid_sync(nd, sync, (unsigned int)(nb * (k + 1)), &s_flag, &s_ev, &nd.stats[2 + ((t + 1) & 1)]))
            break;
    }
    for (int64_t i = threadIdx.x; i < rr.n_cnt; i += blockDim.x) {
        const int64_t id = rr.n_lo + i;
        if (id < nd.N) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < nst) gst[k][id] = st[k][i];
        }
    }
    if (b == 0 && threadIdx.x == 0) *clock = t0 + len;
}

// ---- device generator (fixed fan-out), one warp per row
struct GenDev {
    int64_t src_begin, src_count, tgt_begin, tgt_count;
    int32_t fanout, exclude_self;
    float w_lo, w_hi, w_sign;
    int32_t d_lo, d_hi;
    uint32_t stream;
    uint64_t syn_offset;
    uint32_t k0, k1;
};

struct GenDraw { int64_t t; float w; int m; };

__device__ __forceinline__ GenDraw gen_draw(const GenDev& g, int64_t s, int k)
{
    uint4 x = sz_philox((uint32_t)(s - g.src_begin), (uint32_t)k, g.stream, SZ_STREAM_GEN, g.k0, g.k1);
    GenDraw d;
    if (g.exclude_self && s >= g.tgt_begin && s < g.tgt_begin + g.tgt_count) {
        d.t = g.tgt_begin + sz_bounded(x.x, (uint32_t)(g.tgt_count - 1));
        if (d.t >= s) d.t += 1;
    } else {
        d.t = g.tgt_begin + sz_bounded(x.x, (uint32_t)g.tgt_count);
    }
    float span = g.w_hi - g.w_lo;
    float mag = g.w_lo + span * sz_u24(x.y);
    d.w = g.w_sign * mag;
    d.m = g.d_lo + (int)sz_bounded(x.z, (uint32_t)(g.d_hi - g.d_lo + 1));
    return d;
}

__global__ void __launch_bounds__(256) k_generate(GenDev g, int D, unsigned long long* row_ptr, int2* syn)
{
    extern __shared__ uint32_t s_hist[];
    const uint32_t lane = threadIdx.x & 31;
    uint32_t* h = s_hist + (threadIdx.x >> 5) * D;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int F = g.fanout;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < g.src_count; r += nwarps) {
        const int64_t s = g.src_begin + r;
        const unsigned long long base = g.syn_offset + (unsigned long long)r * (unsigned long long)F;
        for (int j = lane; j < D; j += 32) h[j] = 0;
        __syncwarp();
        for (int k = lane; k < F; k += 32) {
            uint4 x = sz_philox((uint32_t)r, (uint32_t)k, g.stream, SZ_STREAM_GEN, g.k0, g.k1);
            int m = g.d_lo + (int)sz_bounded(x.z, (uint32_t)(g.d_hi - g.d_lo + 1));
            atomicAdd(&h[m - 1], 1u);
        }
        __syncwarp();
        uint32_t carry = 0;
        for (int j0 = 0; j0 < D; j0 += 32) {
            int j = j0 + (int)lane;
            uint32_t c = (j < D) ? h[j] : 0u;
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += y;
            }
            if (j < D) {
                h[j] = carry + incl - c;
                row_ptr[s * D + j] = base + carry + incl - c;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncwarp();
        for (int kb = 0; kb < F; kb += 32) {
            const int k = kb + (int)lane;
            const bool valid = k < F;
            const uint32_t mask = __ballot_sync(0xffffffffu, valid);
            GenDraw d{0, 0.0f, 1};
            uint32_t peers = 0, rank = 0;
            if (valid) {
                d = gen_draw(g, s, k);
                peers = __match_any_sync(mask, d.m);
                rank = __popc(peers & ((1u << lane) - 1u));
                syn[base + h[d.m - 1] + rank] = make_int2((int)d.t, __float_as_int(d.w));
            }
            __syncwarp();
            if (valid && rank == 0) h[d.m - 1] += __popc(peers);
            __syncwarp();
        }
    }
}

// rp_dm[m * U + u] = row_ptr[u * D + m] for m = 0..D (row_ptr has U * D + 1
// entries: m = D of unit u is the start of unit u+1, or the total)
__global__ void k_rp_transpose(const unsigned long long* __restrict__ row_ptr, int64_t U, int D,
                               unsigned long long* __restrict__ rp_dm)
{
    const int64_t n = (int64_t)(D + 1) * U;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = i / U, u = i - m * U;
        rp_dm[i] = row_ptr[u * D + m];
    }
}

__global__ void k_fill_rows(unsigned long long* row_ptr, int64_t s0, int64_t s1, int D, unsigned long long v)
{
    for (int64_t i = s0 * D + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s1 * D;
         i += (int64_t)gridDim.x * blockDim.x)
        row_ptr[i] = v;
}

__global__ void k_check_finite(const float* a, int64_t n, uint32_t* flag)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(a[i])) { *flag = 1u; }
}

__global__ void k_pack_syn(const int32_t* tgt, const float* w, int2* syn, uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        syn[i] = make_int2(tgt[i], __float_as_int(w[i]));
}

__global__ void k_unpack_syn(const int2* syn, int32_t* tgt, float* w, uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        int2 v = syn[i];
        tgt[i] = v.x;
        w[i] = __int_as_float(v.y);
    }
}

int num_sms(szsnn_ctx* ctx) { return ctx->num_sms > 0 ? ctx->num_sms : 148; }

// Units per update thread: UPD_UPT (bulk-copied tiles, fewer and longer
// blocks) only while the update grid still holds at least four blocks per SM;
// smaller networks keep one unit per thread, where the step is latency-bound
// and more blocks in parallel shorten it.
int upd_upt(const szsnn_net* n)
{
    if (n->upd_units > 0) return n->upd_units;
    const int64_t per_sm = sz_div_up(n->U, (int64_t)num_sms(n->ctx) * n->upd_block);  // blocks per SM at 1 unit
    return (int)std::max<int64_t>(1, std::min<int64_t>(UPD_UPT, per_sm / 4));
}

// par: parity of the step counter when the launches built from this run
NetDev make_dev(szsnn_net* n, int par)
{
    NetDev d{};
    d.N = n->N; d.U = n->U; d.words = n->words; d.D = n->D; d.npops = n->npops;
    d.pops = n->d_pops; d.row_ptr = n->d_row_ptr; d.rp_dm = n->d_rp_dm; d.syn = n->d_syn;
    d.st0 = n->d_st[0]; d.st1 = n->d_st[1]; d.st2 = n->d_st[2]; d.st3 = n->d_st[3];
    d.in_e = n->d_in_e[0]; d.in_i = n->d_in_i[0]; d.fx_e = n->d_fx_e[0]; d.fx_i = n->d_fx_i[0];
    d.in_e1 = n->d_in_e[1]; d.in_i1 = n->d_in_i[1]; d.fx_e1 = n->d_fx_e[1]; d.fx_i1 = n->d_fx_i[1];
    d.overlap = n->overlap ? 1u : 0u;
    d.acc_mode = n->acc_mode; d.ring_cnt = n->d_ring_cnt; d.ring_ids = n->d_ring_ids;
    d.clock = n->d_clock; d.stats = n->d_stats; d.err = n->ctx->d_err;
    d.dbg_in_e = nullptr; d.dbg_in_i = nullptr;
    d.group = n->d_group; d.group_spikes = n->d_group_spikes;
    d.blk_pop = n->d_blk_pop;
    d.par0 = (uint32_t)(par & 1);
    d.upt = upd_upt(n);
    d.tiles = n->upd_tiles == 2 ? 2u : (n->upd_tiles == 1 && n->npops <= INLINE_POPS) ? 1u : 0u;
    d.own_lo[0] = n->own_hi[0] < 0 ? 0 : n->own_lo[0];
    d.own_hi[0] = n->own_hi[0] < 0 ? n->N : n->own_hi[0];
    d.own_lo[1] = n->own_hi[1] < 0 ? n->N : n->own_lo[1];
    d.own_hi[1] = n->own_hi[1] < 0 ? n->U : n->own_hi[1];
    // parameter-table slots: the populations with shared parameters and a model
    // the inline update covers, each with the update blocks that lie inside it
    if (n->npops <= INLINE_POPS) {
        const int64_t bs = (int64_t)n->upd_block * d.upt;  // units per update block
        for (int i = 0; i < n->npops; ++i) {
            const PopDev& q = n->h_pops[(size_t)i];
            const bool ok = !q.pn && (q.model == SZSNN_IF_CURR_EXP || q.model == SZSNN_IF_COND_EXP ||
                                      q.model == SZSNN_IZHIKEVICH || q.model == SZSNN_POISSON);
            const int64_t lo = sz_div_up(q.begin, bs);                        // first block starting inside
            const int64_t hi = q.end >= n->U ? sz_div_up(n->U, bs) : q.end / bs;  // blocks ending inside
            if (ok && d.tiles == 1) { d.ipop[i] = q; continue; }  // warp tiles find their slot by unit range
            if (!ok || hi <= lo) continue;
            d.ipop[i] = q;
            d.ib_lo[i] = (int32_t)lo;
            d.ib_hi[i] = (int32_t)hi;
        }
    }
    return d;
}

NetDev make_dev(szsnn_net* n) { return make_dev(n, (int)(n->steps_done & 1)); }

// delivery of delays m_lo..D into the inputs of step clock + k_off
cudaError_t launch_propagate(szsnn_net* n, const NetDev& d, int k_off, int m_lo, uint32_t pf, cudaStream_t st)
{
    int blocks = n->prop_blocks > 0 ? n->prop_blocks : num_sms(n->ctx) * 16;
    if (n->prop_mode == 1) {
        const size_t sm = far_window_bytes(256);
        switch (n->prop_group) {
        case 8: k_propagate_flat<8><<<blocks, 256, sm, st>>>(d, k_off, m_lo, pf); break;
        case 16: k_propagate_flat<16><<<blocks, 256, sm, st>>>(d, k_off, m_lo, pf); break;
        default: k_propagate_flat<32><<<blocks, 256, sm, st>>>(d, k_off, m_lo, pf); break;
        }
        return cudaGetLastError();
    }
    switch (n->prop_group) {
    case 4: k_propagate<4><<<blocks, 256, 0, st>>>(d, k_off, m_lo, pf); break;
    case 8: k_propagate<8><<<blocks, 256, 0, st>>>(d, k_off, m_lo, pf); break;
    case 32: k_propagate<32><<<blocks, 256, 0, st>>>(d, k_off, m_lo, pf); break;
    default: k_propagate<16><<<blocks, 256, 0, st>>>(d, k_off, m_lo, pf); break;
    }
    return cudaGetLastError();
}

// classic order: all delays into step t's (single) buffer, slot t emptied
cudaError_t launch_propagate_classic(szsnn_net* n, const NetDev& d, int k_off, cudaStream_t st)
{
    return launch_propagate(n, d, k_off, 1, PF_ZERO_SLOT | PF_SPIKES, st);
}

// overlapped order: delays 2..D into the parity buffer of step clock + k_off
cudaError_t launch_propagate_far(szsnn_net* n, const NetDev& d, int k_off, cudaStream_t st)
{
    if (n->D < 2) return cudaSuccess;
    return launch_propagate(n, d, k_off, 2, PF_PENDING, st);
}

// (first pop, count) overlapping the tile of each update block
cudaError_t fill_blk_pop(szsnn_net* n)
{
    if (n->npops <= UPD_BLOCK_POPS) return cudaSuccess;
    const int64_t bs = (int64_t)n->upd_block * upd_upt(n);  // units per update block (its tile)
    const int64_t nb = sz_div_up(n->U, bs);
    std::vector<int2> t((size_t)nb);
    int first = 0;
    for (int64_t b = 0; b < nb; ++b) {
        const int64_t b0 = b * bs, b1 = b0 + bs;
        while (first < n->npops && n->pops[(size_t)first].end <= b0) ++first;
        int c = 0;
        for (int i = first; i < n->npops && n->pops[(size_t)i].begin < b1; ++i) ++c;
        t[(size_t)b] = make_int2(first, c);
    }
    if (!n->d_blk_pop) {
        cudaError_t e = cudaMalloc((void**)&n->d_blk_pop, (size_t)sz_div_up(n->U, 32) * sizeof(int2));
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaMemcpyAsync(n->d_blk_pop, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice, n->ctx->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(n->ctx->stream);
}

// dynamic shared memory of an update launch: an inline tile when any block
// of the launch runs one, at least `floor` bytes (the delivery blocks' copy
// windows in a fused step); the kernel's limit raised when above 48 KB
template <class K>
cudaError_t update_smem(const NetDev& d, int bs, K kernel, size_t* bytes, size_t floor = 0)
{
    bool any = false;
    for (int i = 0; i < INLINE_POPS; ++i) any = any || d.ib_hi[i] > d.ib_lo[i];
    *bytes = any ? tile_smem_bytes((int64_t)d.upt * bs, d.acc_mode == SZSNN_ACC_FIXED) : 0;
    if (d.tiles == 1) *bytes = (size_t)(bs / 32) * wt_region_bytes(d.acc_mode == SZSNN_ACC_FIXED);
    *bytes = std::max(*bytes, floor);
    if (*bytes > 48 * 1024)
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*bytes);
    return cudaSuccess;
}

// the state monitor's record of step clock + k_off (when a monitor is set)
cudaError_t launch_monitor(szsnn_net* n, const NetDev& d, int k_off, cudaStream_t st)
{
    if (!n->mon_n) return cudaSuccess;
    const int grid = (int)std::min<int64_t>(sz_div_up(n->mon_n, 256), 1024);
    k_monitor<<<grid, 256, 0, st>>>(d.clock, k_off, n->d_mon_t0, d.st0, d.st1, d.st2, d.st3, n->d_mon_ids, n->mon_n,
                                    n->mon_slots, n->d_mon_buf, (long long)n->mon_cap);
    return cudaGetLastError();
}

// update blocks of a launch: one per tile, or the persistent warp-tile grid
// (blocks per SM as tuned, at most one warp per warp tile)
int64_t update_blocks(const szsnn_net* n, const NetDev& d, int bs)
{
    if (d.tiles == 1) {
        const int64_t per_sm = n->upd_per_sm > 0 ? n->upd_per_sm : 2;
        return std::max<int64_t>(1, std::min<int64_t>(sz_div_up(sz_div_up(n->U, WT), bs / 32),
                                                      per_sm * num_sms(n->ctx)));
    }
    return sz_div_up(n->U, (int64_t)bs * d.upt);
}

// persistent block tiles: as many update blocks as stay resident beside the
// `far` delivery blocks (or the tuned count per SM), at most one per tile
template <class K>
int64_t persistent_blocks(const szsnn_net* n, const NetDev& d, K kernel, int bs, size_t smem, int64_t far)
{
    const int64_t sms = num_sms(n->ctx), tiles = sz_div_up(n->U, (int64_t)bs * d.upt);
    int64_t total;
    if (n->upd_per_sm > 0) {
        total = (int64_t)n->upd_per_sm * sms;
    } else {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, bs, smem) != cudaSuccess || occ < 1) {
            cudaGetLastError();
            occ = 1;
        }
        total = std::max<int64_t>(sms, occ * sms - far);
    }
    return std::max<int64_t>(1, std::min<int64_t>(total, tiles));
}

template <int MODE>
cudaError_t launch_update_mode(szsnn_net* n, const NetDev& d, int k_off, const uint32_t* forced, const float* cur,
                               uint32_t* words, cudaStream_t st)
{
    const int bs = n->upd_block;
    size_t smem = 0;
    cudaError_t e = update_smem(d, bs, k_update<MODE>, &smem);
    if (e != cudaSuccess) return e;
    const int64_t blocks = MODE == 2 ? persistent_blocks(n, d, k_update<MODE>, bs, smem, 0) : update_blocks(n, d, bs);
    k_update<MODE><<<(unsigned)blocks, bs, smem, st>>>(d, k_off, forced, cur, words);
    return cudaGetLastError();
}

cudaError_t launch_update(szsnn_net* n, const NetDev& d, int k_off, const uint32_t* forced, const float* cur,
                          uint32_t* words, cudaStream_t st)
{
    if (d.tiles == 1) return launch_update_mode<1>(n, d, k_off, forced, cur, words, st);
    if (d.tiles == 2) return launch_update_mode<2>(n, d, k_off, forced, cur, words, st);
    return launch_update_mode<0>(n, d, k_off, forced, cur, words, st);
}


// overlapped step clock + k_off: far delivery into step t+1 and update(t) in one launch
cudaError_t launch_step(szsnn_net* n, const NetDev& d, int k_off, const uint32_t* forced, const float* cur,
                        uint32_t* words, cudaStream_t st)
{
    const int bs = n->upd_block;
    const int far = n->D < 2 ? 0 : (n->prop_blocks > 0 ? n->prop_blocks : num_sms(n->ctx) * std::max(1, 1024 / bs));
    const size_t win = (far > 0 && n->prop_mode == 1) ? far_window_bytes(bs) : 0;
    size_t smem = 0;
    cudaError_t e = cudaSuccess;
#define SZ_STEP_MODE(G, M)                                                                                     \
    do {                                                                                                      \
        e = update_smem(d, bs, k_step<G, M>, &smem, win);                                                     \
        if (e != cudaSuccess) break;                                                                          \
        const int64_t ub = M == 2 ? persistent_blocks(n, d, k_step<G, M>, bs, smem, far) : update_blocks(n, d, bs); \
        k_step<G, M><<<(unsigned)(far + ub), bs, smem, st>>>(d, k_off, far, forced, cur, words);             \
    } while (0)
#define SZ_STEP(G)                                        \
    do {                                                  \
        if (d.tiles == 1) SZ_STEP_MODE(G, 1);             \
        else if (d.tiles == 2) SZ_STEP_MODE(G, 2);        \
        else SZ_STEP_MODE(G, 0);                          \
    } while (0)
    if (n->prop_mode == 1) {
        switch (n->prop_group) {
        case 8: SZ_STEP(-8); break;
        case 16: SZ_STEP(-16); break;
        default: SZ_STEP(-32); break;
        }
    } else {
        switch (n->prop_group) {
        case 4: SZ_STEP(4); break;
        case 8: SZ_STEP(8); break;
        case 32: SZ_STEP(32); break;
        default: SZ_STEP(16); break;
        }
    }
#undef SZ_STEP
#undef SZ_STEP_MODE
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// ---- resident stepping (host)

int res_blocks(const szsnn_net* n)
{
    const int64_t want = n->res_blocks > 0 ? n->res_blocks : num_sms(n->ctx);
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, n->words));
}

template <bool FIXED>
void* res_kernel(int ipw)
{
    if (ipw == 8) return (void*)k_resident<FIXED, 8>;
    if (ipw == 32) return (void*)k_resident<FIXED, 32>;
    return (void*)k_resident<FIXED, 16>;
}

void* res_kernel(const szsnn_net* n)
{
    const int ipw = n->prop_mode == 1 ? n->prop_group : 16;
    return n->acc_mode == SZSNN_ACC_FIXED ? res_kernel<true>(ipw) : res_kernel<false>(ipw);
}

// Whether the network can step resident; on success the dynamic shared
// memory and the state slots kept.  `why` names the first obstacle.
bool res_check(szsnn_net* n, std::string* why, size_t* smem, int* nst)
{
    auto no = [&](const char* m) { if (why) *why = m; return false; };
    if (!n->overlap) return no("resident stepping needs the overlapped step order");
    if (n->npops > INLINE_POPS) return no("resident stepping takes at most 4 populations");
    if (n->mon_n) return no("resident stepping does not record a state monitor");
    if (n->res_uw < 1 || n->res_uw > RES_THREADS / 32 - 1) return no("update warps must be in 1..31");
    if (n->U >= ((int64_t)1 << 31)) return no("resident stepping takes fewer than 2^31 units");
    int slots = 2;
    for (const PopDev& q : n->h_pops) {
        const bool neuron_model = q.model == SZSNN_IF_CURR_EXP || q.model == SZSNN_IF_COND_EXP ||
                                  q.model == SZSNN_IZHIKEVICH;
        if (q.begin < n->N && q.end > n->N) return no("a population spans neurons and sources");
        if (q.begin < n->N && !neuron_model) return no("neurons of a source model");
        if (q.begin >= n->N && q.model != SZSNN_POISSON) return no("sources other than Poisson");
        if (q.model != SZSNN_IZHIKEVICH && neuron_model) slots = 4;
    }
    int dev = 0, coop = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return no("device attributes unavailable");
    }
    if (!coop) return no("the device has no cooperative launch");
    const int nb = res_blocks(n);
    const size_t bytes = (size_t)(RES_THREADS / 32 - n->res_uw) * 32 * FAR_WPL * sizeof(int2) +
                         (size_t)slots * (size_t)res_cap(n->N, nb) * sizeof(float);
    void* k = res_kernel(n);
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) { cudaGetLastError(); return no("kernel attributes unavailable"); }
    if (bytes + fa.sharedSizeBytes > (size_t)optin)
        return no("the neuron state of a block does not fit in shared memory");
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) {
        cudaGetLastError();
        return no("shared memory limit not accepted");
    }
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, RES_THREADS, bytes) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        return no("a resident block does not fit on an SM");
    }
    if ((int64_t)occ * num_sms(n->ctx) < nb) return no("more resident blocks than fit on the device");
    *smem = bytes;
    *nst = slots;
    return true;
}

// one chunk of `len` resident steps (stage buffer b of the run's I/O);
// smem and nst from res_check
cudaError_t launch_resident(szsnn_net* n, int len, int flags, int b, cudaStream_t st, size_t smem, int nst)
{
    if (!n->d_res_sync) {
        cudaError_t e = cudaMalloc((void**)&n->d_res_sync, sizeof(ResSync));
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaMemsetAsync(n->d_res_sync, 0, sizeof(ResSync), st);
    if (e != cudaSuccess) return e;
    NetDev d = make_dev(n, 0);
    ResSync* sync = reinterpret_cast<ResSync*>(n->d_res_sync);
    long long* clock = n->d_clock;
    const uint32_t* fw = (flags & 1) ? n->d_forced_stage[b] : nullptr;
    const float* cu = (flags & 2) ? n->d_current_stage : nullptr;
    uint32_t* ras = (flags & 4) ? n->d_raster_stage[b] : nullptr;
    int uw = n->res_uw;
    void* args[] = {&d, &sync, &clock, &len, &uw, &nst, &fw, &cu, &ras};
    return cudaLaunchCooperativeKernel(res_kernel(n), dim3((unsigned)res_blocks(n)), dim3(RES_THREADS), args, smem, st);
}

template <class T>
cudaError_t dalloc(T** p, size_t count)
{
    *p = nullptr;
    count = (count + 31) & ~(size_t)31;  // room for bulk copies rounded up to 16 bytes
    if (!count) count = 32;
    return cudaMalloc((void**)p, count * sizeof(T));
}

void free_net(szsnn_net* n)
{
    if (!n) return;
    for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);
    n->graphs.clear();
    cudaFree(n->d_pops);
    cudaFree(n->d_pn);
    cudaFree(n->d_group);
    cudaFree(n->d_group_spikes);
    cudaFree(n->d_blk_pop);
    cudaFree(n->d_row_ptr);
    cudaFree(n->d_rp_dm);
    cudaFree(n->d_mon_ids);
    cudaFree(n->d_mon_buf);
    cudaFree(n->d_mon_t0);
    cudaFree(n->d_syn);
    for (int k = 0; k < 4; ++k) cudaFree(n->d_st[k]);
    for (int p = 0; p < 2; ++p) {
        cudaFree(n->d_in_e[p]);
        cudaFree(n->d_in_i[p]);
        cudaFree(n->d_fx_e[p]);
        cudaFree(n->d_fx_i[p]);
        cudaFree(n->d_forced_stage[p]);
        cudaFree(n->d_raster_stage[p]);
    }
    cudaFree(n->d_ring_cnt);
    cudaFree(n->d_ring_ids);
    cudaFree(n->d_clock);
    cudaFree(n->d_stats);
    cudaFree(n->d_current_stage);
    cudaFree(n->d_dbg_in);
    cudaFree(n->d_inject);
    cudaFree(n->d_res_sync);
    if (n->h_pinned_words) cudaFreeHost(n->h_pinned_words);
    for (auto& h : n->h_io) if (h) cudaFreeHost(h);
    if (n->ev_run0) cudaEventDestroy(n->ev_run0);
    if (n->ev_run1) cudaEventDestroy(n->ev_run1);
    for (int p = 0; p < 2; ++p)
        for (cudaEvent_t ev : {n->ev_in[p], n->ev_comp[p], n->ev_out[p]}) if (ev) cudaEventDestroy(ev);
    if (n->copy_st) cudaStreamDestroy(n->copy_st);
    if (n->copy_out_st) cudaStreamDestroy(n->copy_out_st);
    delete n;
}

}  // namespace

#define NET_TRY(n, call)                                                                        \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return szsnn_set_error((n)->ctx, e_ == cudaErrorMemoryAllocation ? SZSNN_ERR_NOMEM   \
                                                                            : SZSNN_ERR_CUDA,   \
                                   std::string(#call) + ": " + cudaGetErrorString(e_));         \
    } while (0)

// the delay-major copy of row_ptr, rebuilt whenever the synapses change
static cudaError_t build_rp_dm(szsnn_net* n)
{
    cudaStream_t st = n->ctx->stream;
    if (!n->d_rp_dm) {
        cudaError_t e = dalloc(&n->d_rp_dm, (size_t)(n->D + 1) * (size_t)n->U);
        if (e != cudaSuccess) return e;
    }
    k_rp_transpose<<<num_sms(n->ctx) * 8, 256, 0, st>>>(n->d_row_ptr, n->U, n->D, n->d_rp_dm);
    return cudaGetLastError();
}

extern "C" int szsnn_net_create(szsnn_ctx* ctx, const szsnn_net_desc* d, szsnn_net** out)
{
    if (!ctx || !d || !out) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_net_create: null argument");
    *out = nullptr;
    if (d->n_neurons < 0 || d->n_sources < 0 || d->n_neurons + d->n_sources < 1)
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_net_create: no units");
    if (d->n_neurons + d->n_sources > 0x7fffffffLL)
        return szsnn_set_error(ctx, SZSNN_ERR_LIMIT, "szsnn_net_create: more than 2^31-1 units");
    if (d->max_delay < 1 || d->max_delay > 1024)
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_net_create: max_delay outside 1..1024");
    if (d->n_pops < 0 || d->n_pops > SZSNN_MAX_POPS || (d->n_pops > 0 && !d->pops))
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_net_create: bad population table");
    if (d->group_host && (d->n_groups < 1))
        return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_net_create: group_host needs n_groups >= 1");
    if (d->acc_mode > 1) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "szsnn_net_create: bad acc_mode");
    const int64_t N = d->n_neurons, U = d->n_neurons + d->n_sources;
    for (int i = 0; i < d->n_pops; ++i) {
        const szsnn_pop_desc& p = d->pops[i];
        if (p.begin < 0 || p.end > U || p.begin > p.end)
            return szsnn_set_error(ctx, SZSNN_ERR_ARG, "pop " + std::to_string(i) + ": range outside the units");
        bool neuron_model = p.model == SZSNN_IF_CURR_EXP || p.model == SZSNN_IF_COND_EXP || p.model == SZSNN_IZHIKEVICH;
        bool source_model = p.model == SZSNN_POISSON || p.model == SZSNN_CONST_RATE;
        if (!neuron_model && !source_model)
            return szsnn_set_error(ctx, SZSNN_ERR_ARG, "pop " + std::to_string(i) + ": unknown model");
        if (p.begin < p.end && neuron_model && p.end > N)
            return szsnn_set_error(ctx, SZSNN_ERR_ARG, "pop " + std::to_string(i) + ": neuron model on source ids");
        if (p.begin < p.end && source_model && p.begin < N)
            return szsnn_set_error(ctx, SZSNN_ERR_ARG, "pop " + std::to_string(i) + ": source model on neuron ids");
        if (i > 0 && p.begin < d->pops[i - 1].end)
            return szsnn_set_error(ctx, SZSNN_ERR_ARG,
                                   "pops " + std::to_string(i - 1) + " and " + std::to_string(i) + " overlap or are not sorted");
    }
    const int D = d->max_delay;
    if (d->row_ptr_host) {  // host CSR: bucket pointers must be monotone and end at n_synapses
        const uint64_t* rp = d->row_ptr_host;
        const uint64_t cnt = (uint64_t)U * D;
        if (rp[0] != 0 || rp[cnt] != d->n_synapses)
            return szsnn_set_error(ctx, SZSNN_ERR_ARG, "row_ptr must start at 0 and end at n_synapses");
        for (uint64_t i = 0; i < cnt; ++i)
            if (rp[i + 1] < rp[i]) return szsnn_set_error(ctx, SZSNN_ERR_ARG, "row_ptr not monotone");
        if (d->n_synapses && (!d->tgt_host || !d->w_host))
            return szsnn_set_error(ctx, SZSNN_ERR_ARG, "tgt/w missing");
    }

    szsnn_net* n = new szsnn_net();
    n->ctx = ctx;
    n->N = N; n->U = U; n->words = sz_div_up(U, 32); n->D = D; n->R = D + 1;
    n->acc_mode = d->acc_mode; n->npops = d->n_pops;
    n->chunk = d->graph_chunk ? (int)d->graph_chunk : 100;
    n->n_syn = d->n_synapses;
    n->pops.assign(d->pops, d->pops + d->n_pops);
    cudaStream_t st = ctx->stream;
#define C(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { std::string m_ = std::string(#x) + ": " + cudaGetErrorString(e_); int code_ = e_ == cudaErrorMemoryAllocation ? SZSNN_ERR_NOMEM : SZSNN_ERR_CUDA; free_net(n); return szsnn_set_error(ctx, code_, m_); } } while (0)
    // populations; per-unit parameter arrays packed into one device buffer
    {
        std::vector<PopDev> hp((size_t)std::max(d->n_pops, 1));
        size_t pn_total = 0;
        for (int i = 0; i < d->n_pops; ++i)
            if (d->pops[i].pn_host && d->pops[i].end > d->pops[i].begin)
                pn_total += (size_t)POP_SLOTS * (d->pops[i].end - d->pops[i].begin);
        if (pn_total) C(dalloc(&n->d_pn, pn_total));
        size_t off = 0;
        std::vector<float> tmp;
        for (int i = 0; i < d->n_pops; ++i) {
            const szsnn_pop_desc& p = d->pops[i];
            PopDev& q = hp[(size_t)i];
            std::memset(&q, 0, sizeof(q));
            q.model = p.model; q.flags = p.flags; q.begin = p.begin; q.end = p.end;
            std::memcpy(q.p, p.p, sizeof(p.p));
            const bool if_model = p.model == SZSNN_IF_CURR_EXP || p.model == SZSNN_IF_COND_EXP;
            if (if_model) { q.p[12] = sz_decay(p.p[4]); q.p[13] = sz_decay(p.p[5]); }
            q.seed = p.seed;
            if (p.pn_host && p.end > p.begin) {
                const size_t cnt = (size_t)(p.end - p.begin);
                tmp.assign((size_t)POP_SLOTS * cnt, 0.0f);
                std::memcpy(tmp.data(), p.pn_host, 12 * cnt * sizeof(float));
                if (if_model)
                    for (size_t u = 0; u < cnt; ++u) {
                        tmp[12 * cnt + u] = sz_decay(tmp[4 * cnt + u]);
                        tmp[13 * cnt + u] = sz_decay(tmp[5 * cnt + u]);
                    }
                C(cudaMemcpy(n->d_pn + off, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice));
                q.pn = n->d_pn + off;
                off += tmp.size();
            }
        }
        n->h_pops = hp;
        C(dalloc(&n->d_pops, hp.size()));
        C(cudaMemcpyAsync(n->d_pops, hp.data(), hp.size() * sizeof(PopDev), cudaMemcpyHostToDevice, st));
        C(cudaStreamSynchronize(st));
    }
    C(fill_blk_pop(n));
    if (d->group_host) {
        for (int64_t i = 0; i < U; ++i)
            if (d->group_host[i] < 0 || d->group_host[i] >= d->n_groups) {
                free_net(n);
                return szsnn_set_error(ctx, SZSNN_ERR_ARG, "group id outside 0..n_groups-1");
            }
        n->n_groups = d->n_groups;
        C(dalloc(&n->d_group, (size_t)U));
        C(cudaMemcpyAsync(n->d_group, d->group_host, (size_t)U * 4, cudaMemcpyHostToDevice, st));
        C(dalloc(&n->d_group_spikes, (size_t)d->n_groups));
        C(cudaMemsetAsync(n->d_group_spikes, 0, (size_t)d->n_groups * 8, st));
    }
    // synapses
    C(dalloc(&n->d_row_ptr, (size_t)U * D + 1));
    C(dalloc(&n->d_syn, (size_t)n->n_syn));
    if (d->row_ptr_host) {
        C(cudaMemcpyAsync(n->d_row_ptr, d->row_ptr_host, ((size_t)U * D + 1) * 8, cudaMemcpyHostToDevice, st));
        if (n->n_syn) {  // pack tgt/w into {int32, fp32} pairs in bounded chunks
            const uint64_t CH = 1ull << 26;
            int32_t* dt = nullptr;
            float* dw = nullptr;
            C(dalloc(&dt, (size_t)std::min<uint64_t>(CH, n->n_syn)));
            C(dalloc(&dw, (size_t)std::min<uint64_t>(CH, n->n_syn)));
            for (uint64_t o = 0; o < n->n_syn; o += CH) {
                uint64_t c = std::min<uint64_t>(CH, n->n_syn - o);
                C(cudaMemcpyAsync(dt, d->tgt_host + o, c * 4, cudaMemcpyHostToDevice, st));
                C(cudaMemcpyAsync(dw, d->w_host + o, c * 4, cudaMemcpyHostToDevice, st));
                k_pack_syn<<<1024, 256, 0, st>>>(dt, dw, n->d_syn + o, c);
                C(cudaGetLastError());
            }
            C(cudaStreamSynchronize(st));
            cudaFree(dt);
            cudaFree(dw);
        }
    } else {
        C(cudaMemsetAsync(n->d_row_ptr, 0, ((size_t)U * D + 1) * 8, st));
    }
    C(build_rp_dm(n));
    // state
    for (int k = 0; k < 4; ++k) {
        C(dalloc(&n->d_st[k], (size_t)U));
        if (d->state_host[k]) C(cudaMemcpyAsync(n->d_st[k], d->state_host[k], (size_t)U * 4, cudaMemcpyHostToDevice, st));
        else C(cudaMemsetAsync(n->d_st[k], 0, (size_t)U * 4, st));
    }
    const size_t N1 = (size_t)std::max<int64_t>(N, 1);
    for (int p = 0; p < 2; ++p) {
        C(dalloc(&n->d_in_e[p], N1)); C(cudaMemsetAsync(n->d_in_e[p], 0, N1 * 4, st));
        C(dalloc(&n->d_in_i[p], N1)); C(cudaMemsetAsync(n->d_in_i[p], 0, N1 * 4, st));
        if (n->acc_mode == SZSNN_ACC_FIXED) {
            C(dalloc(&n->d_fx_e[p], N1)); C(cudaMemsetAsync(n->d_fx_e[p], 0, N1 * 8, st));
            C(dalloc(&n->d_fx_i[p], N1)); C(cudaMemsetAsync(n->d_fx_i[p], 0, N1 * 8, st));
        }
    }
    C(dalloc(&n->d_ring_cnt, (size_t)n->R)); C(cudaMemsetAsync(n->d_ring_cnt, 0, (size_t)n->R * 4, st));
    C(dalloc(&n->d_ring_ids, (size_t)n->R * U));
    C(dalloc(&n->d_clock, 1)); C(cudaMemsetAsync(n->d_clock, 0, 8, st));
    C(dalloc(&n->d_stats, 4)); C(cudaMemsetAsync(n->d_stats, 0, 32, st));
    for (int p = 0; p < 2; ++p) {
        C(dalloc(&n->d_forced_stage[p], (size_t)n->chunk * n->words));
        C(dalloc(&n->d_raster_stage[p], (size_t)n->chunk * n->words));
    }
    C(dalloc(&n->d_current_stage, (size_t)n->chunk * std::max<int64_t>(N, 1)));
    C(dalloc(&n->d_dbg_in, (size_t)2 * std::max<int64_t>(N, 1)));
    C(cudaMallocHost((void**)&n->h_pinned_words, (size_t)n->words * 4));
    C(cudaEventCreate(&n->ev_run0));
    C(cudaEventCreate(&n->ev_run1));
    C(cudaStreamCreateWithFlags(&n->copy_st, cudaStreamNonBlocking));
    C(cudaStreamCreateWithFlags(&n->copy_out_st, cudaStreamNonBlocking));
    for (int p = 0; p < 2; ++p) {
        C(cudaEventCreateWithFlags(&n->ev_in[p], cudaEventDisableTiming));
        C(cudaEventCreateWithFlags(&n->ev_comp[p], cudaEventDisableTiming));
        C(cudaEventCreateWithFlags(&n->ev_out[p], cudaEventDisableTiming));
    }
    C(cudaStreamSynchronize(st));
#undef C
    *out = n;
    return SZSNN_OK;
}

extern "C" int szsnn_net_destroy(szsnn_net* n)
{
    if (!n) return SZSNN_ERR_ARG;
    cudaStreamSynchronize(n->ctx->stream);
    free_net(n);
    return SZSNN_OK;
}

extern "C" int szsnn_net_generate(szsnn_net* n, const szsnn_gen_block* blocks, int nb, uint64_t seed)
{
    if (!n || (nb > 0 && !blocks) || nb < 0) return szsnn_set_error(n ? n->ctx : nullptr, SZSNN_ERR_ARG, "szsnn_net_generate: bad arguments");
    cudaStream_t st = n->ctx->stream;
    const int D = n->D;
    // blocks must be sorted by src_begin and disjoint; synapse offsets are cumulative
    uint64_t off = 0;
    int64_t row = 0;
    for (int i = 0; i < nb; ++i) {
        const szsnn_gen_block& b = blocks[i];
        if (b.src_begin < row || b.src_count < 0 || b.src_begin + b.src_count > n->U || b.fanout < 0 ||
            b.d_lo < 1 || b.d_hi > D || b.d_lo > b.d_hi || b.tgt_begin < 0 || b.tgt_count < 1 ||
            b.tgt_begin + b.tgt_count > n->N || (b.exclude_self && b.tgt_count < 2))
            return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "szsnn_net_generate: bad block " + std::to_string(i));
        if (b.src_begin > row) {
            k_fill_rows<<<256, 256, 0, st>>>(n->d_row_ptr, row, b.src_begin, D, off);
            NET_TRY(n, cudaGetLastError());
        }
        off += (uint64_t)b.src_count * (uint64_t)b.fanout;
        row = b.src_begin + b.src_count;
    }
    if (row < n->U) {
        k_fill_rows<<<256, 256, 0, st>>>(n->d_row_ptr, row, n->U, D, off);
        NET_TRY(n, cudaGetLastError());
    }
    if (off != n->n_syn) {  // (re)allocate synapse storage for the generated count
        NET_TRY(n, cudaStreamSynchronize(st));
        for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);  // they hold the old array
        n->graphs.clear();
        cudaFree(n->d_syn);
        n->d_syn = nullptr;
        NET_TRY(n, dalloc(&n->d_syn, (size_t)off));
        n->n_syn = off;
    }
    const unsigned long long total = off;
    NET_TRY(n, cudaMemcpyAsync(n->d_row_ptr + (size_t)n->U * D, &total, 8, cudaMemcpyHostToDevice, st));
    off = 0;
    const size_t smem = (size_t)8 * D * 4;
    if (smem > 48 * 1024) NET_TRY(n, cudaFuncSetAttribute(k_generate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (int i = 0; i < nb; ++i) {
        const szsnn_gen_block& b = blocks[i];
        GenDev g{b.src_begin, b.src_count, b.tgt_begin, b.tgt_count, b.fanout, b.exclude_self,
                 b.w_lo, b.w_hi, b.w_sign, b.d_lo, b.d_hi, b.stream, off,
                 (uint32_t)seed, (uint32_t)(seed >> 32)};
        if (b.src_count > 0) {
            int64_t blocks_needed = sz_div_up(b.src_count, 8);
            int grid = (int)std::min<int64_t>(blocks_needed, (int64_t)num_sms(n->ctx) * 16);
            k_generate<<<grid, 256, smem, st>>>(g, D, n->d_row_ptr, n->d_syn);
            NET_TRY(n, cudaGetLastError());
        }
        off += (uint64_t)b.src_count * (uint64_t)b.fanout;
    }
    NET_TRY(n, build_rp_dm(n));
    NET_TRY(n, cudaStreamSynchronize(st));
    return SZSNN_OK;
}

static int net_stage_step_inputs(szsnn_net* n, const uint32_t* forced_host, const float* current_host)
{
    cudaStream_t st = n->ctx->stream;
    if (forced_host)
        NET_TRY(n, cudaMemcpyAsync(n->d_forced_stage[0], forced_host, (size_t)n->words * 4, cudaMemcpyHostToDevice, st));
    if (current_host && n->N)
        NET_TRY(n, cudaMemcpyAsync(n->d_current_stage, current_host, (size_t)n->N * 4, cudaMemcpyHostToDevice, st));
    return SZSNN_OK;
}

extern "C" int szsnn_net_step(szsnn_net* n, const uint32_t* forced_host, const float* current_host,
                              uint32_t* fired_host)
{
    if (!n) return SZSNN_ERR_ARG;
    int rc = net_stage_step_inputs(n, forced_host, current_host);
    if (rc) return rc;
    NetDev d = make_dev(n);
    d.dbg_in_e = n->d_dbg_in;
    d.dbg_in_i = n->d_dbg_in + std::max<int64_t>(n->N, 1);
    cudaStream_t st = n->ctx->stream;
    const uint32_t* forced = forced_host ? n->d_forced_stage[0] : nullptr;
    const float* cur = current_host ? n->d_current_stage : nullptr;
    if (n->overlap) {  // update(t) with its m = 1 deliveries, and delays >= 2 into step t+1
        NET_TRY(n, launch_step(n, d, 0, forced, cur, n->d_raster_stage[0], st));
    } else {
        NET_TRY(n, launch_propagate_classic(n, d, 0, st));
        NET_TRY(n, launch_update(n, d, 0, forced, cur, n->d_raster_stage[0], st));
    }
    NET_TRY(n, launch_monitor(n, d, 0, st));
    k_advance<<<1, 1, 0, st>>>(n->d_clock, 1);
    NET_TRY(n, cudaGetLastError());
    n->kernel_launches += (n->overlap ? 2 : 3) + (n->mon_n ? 1 : 0);
    n->steps_done += 1;
    if (fired_host) {
        NET_TRY(n, cudaMemcpyAsync(n->h_pinned_words, n->d_raster_stage[0], (size_t)n->words * 4, cudaMemcpyDeviceToHost, st));
        NET_TRY(n, cudaStreamSynchronize(st));
        std::memcpy(fired_host, n->h_pinned_words, (size_t)n->words * 4);
    }
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_owned(szsnn_net* n, int64_t n_lo, int64_t n_hi, int64_t s_lo, int64_t s_hi)
{
    if (!n) return SZSNN_ERR_ARG;
    if (n_lo < 0 || n_lo > n_hi || n_hi > n->N || s_lo < n->N || s_lo > s_hi || s_hi > n->U)
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG,
                               "szsnn_net_set_owned: ranges must satisfy 0 <= n_lo <= n_hi <= N <= s_lo <= s_hi <= N+P");
    n->own_lo[0] = n_lo;
    n->own_hi[0] = n_hi;
    n->own_lo[1] = s_lo;
    n->own_hi[1] = s_hi;
    for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);
    n->graphs.clear();
    return SZSNN_OK;
}

extern "C" int szsnn_net_inject_spikes(szsnn_net* n, const uint32_t* words_host)
{
    if (!n || !words_host) return n ? szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "szsnn_net_inject_spikes: null words")
                                    : SZSNN_ERR_ARG;
    if (n->steps_done < 1)
        return szsnn_set_error(n->ctx, SZSNN_ERR_STATE, "szsnn_net_inject_spikes: no step has run yet");
    cudaStream_t st = n->ctx->stream;
    if (!n->d_inject) NET_TRY(n, dalloc(&n->d_inject, (size_t)n->words));
    std::memcpy(n->h_pinned_words, words_host, (size_t)n->words * 4);
    NET_TRY(n, cudaMemcpyAsync(n->d_inject, n->h_pinned_words, (size_t)n->words * 4, cudaMemcpyHostToDevice, st));
    const int grid = (int)std::min<int64_t>(sz_div_up(n->words * 32, 256), (int64_t)num_sms(n->ctx) * 8);
    k_inject<<<grid, 256, 0, st>>>(make_dev(n), n->d_inject);
    NET_TRY(n, cudaGetLastError());
    NET_TRY(n, cudaStreamSynchronize(st));  // the pinned staging buffer is free again on return
    n->kernel_launches += 1;
    return SZSNN_OK;
}

// graph of `len` steps starting at a step of parity `par`; flags bit0
// forced, bit1 current, bit2 raster; `b` selects the forced / raster stage
// buffers.  Overlapped order: one k_step per step (on entry the inputs of the
// first step are complete: its far delivery ran in the previous step's
// launch, or at priming).
static int net_graph(szsnn_net* n, int len, int flags, int b, int par, cudaGraphExec_t* out)
{
    auto key = std::make_tuple(len, flags, b, par & 1);
    auto it = n->graphs.find(key);
    if (it != n->graphs.end()) { *out = it->second; return SZSNN_OK; }
    cudaStream_t st = n->ctx->stream;
    NetDev d = make_dev(n, par);
    cudaGraph_t g = nullptr;
    NET_TRY(n, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < len && e == cudaSuccess; ++k) {
        const uint32_t* fw = (flags & 1) ? n->d_forced_stage[b] + (size_t)k * n->words : nullptr;
        const float* cu = (flags & 2) ? n->d_current_stage + (size_t)k * std::max<int64_t>(n->N, 1) : nullptr;
        uint32_t* ras = (flags & 4) ? n->d_raster_stage[b] + (size_t)k * n->words : nullptr;
        if (n->overlap) {
            e = launch_step(n, d, k, fw, cu, ras, st);
        } else {
            e = launch_propagate_classic(n, d, k, st);
            if (e == cudaSuccess) e = launch_update(n, d, k, fw, cu, ras, st);
        }
        if (e == cudaSuccess) e = launch_monitor(n, d, k, st);
    }
    if (e == cudaSuccess) {
        k_advance<<<1, 1, 0, st>>>(n->d_clock, len);
        e = cudaGetLastError();
    }
    cudaError_t e2 = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return szsnn_set_error(n->ctx, SZSNN_ERR_CUDA,
                               std::string("graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    NET_TRY(n, e);
    n->graphs[key] = ex;
    *out = ex;
    return SZSNN_OK;
}

// Inputs of the next step rebuilt from the ring: both buffers and the pending
// event counters zeroed; in overlapped order all delays (1..D) of step t are
// then delivered into its parity buffer (what far(t) and update(t-1) would
// have delivered), slot t emptied, events counted as pending.  Used after a
// restore and when the step order changes.
static int net_prime(szsnn_net* n)
{
    cudaStream_t st = n->ctx->stream;
    const size_t N1 = (size_t)std::max<int64_t>(n->N, 1);
    for (int p = 0; p < 2; ++p) {
        NET_TRY(n, cudaMemsetAsync(n->d_in_e[p], 0, N1 * 4, st));
        NET_TRY(n, cudaMemsetAsync(n->d_in_i[p], 0, N1 * 4, st));
        if (n->d_fx_e[p]) NET_TRY(n, cudaMemsetAsync(n->d_fx_e[p], 0, N1 * 8, st));
        if (n->d_fx_i[p]) NET_TRY(n, cudaMemsetAsync(n->d_fx_i[p], 0, N1 * 8, st));
    }
    NET_TRY(n, cudaMemsetAsync(n->d_stats + 2, 0, 16, st));
    if (n->overlap) NET_TRY(n, launch_propagate(n, make_dev(n), 0, 1, PF_ZERO_SLOT | PF_PENDING, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_overlap(szsnn_net* n, int on)
{
    if (!n) return SZSNN_ERR_ARG;
    if (on != 0 && on != 1) return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "overlap must be 0 or 1");
    if ((on != 0) == n->overlap) return SZSNN_OK;
    n->overlap = on != 0;
    for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);
    n->graphs.clear();
    return net_prime(n);
}

// true when [p, p + bytes) lies in page-locked host memory (so it can be a
// DMA source / destination without a bounce copy)
static bool host_pinned(const void* p, size_t bytes)
{
    if (!p || !bytes) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    if (a.type != cudaMemoryTypeHost) return false;
    cudaPointerAttributes z{};
    if (cudaPointerGetAttributes(&z, (const char*)p + bytes - 1) != cudaSuccess) { cudaGetLastError(); return false; }
    return z.type == cudaMemoryTypeHost;
}

// Chunks of `chunk` steps, each one graph launch.  Host / device copies of the
// forced words and of the raster run on two copy streams (one per direction)
// into alternating stage buffers, so chunk k+1's input copy and chunk k-1's
// raster copy both overlap chunk k's compute.  Pinned
// host arrays are copied directly; pageable ones go through pinned bounce
// buffers (the copy-out of chunk k to the caller's array happens while chunk
// k+1 runs).
static int net_run_impl(szsnn_net* n, int64_t steps, const uint32_t* forced, const float* current, uint32_t* raster,
                        bool host)
{
    if (!n || steps < 0) return SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream, cp = n->copy_st, cpo = n->copy_out_st;
    const size_t wbytes = (size_t)n->words * 4;
    const bool pin_in = host && forced && host_pinned(forced, (size_t)steps * wbytes);
    const bool pin_out = host && raster && host_pinned(raster, (size_t)steps * wbytes);
    const bool bounce_in = host && forced && !pin_in, bounce_out = host && raster && !pin_out;
    for (int q = 0; q < 4; ++q) {
        const bool need = q < 2 ? bounce_in : bounce_out;
        if (need && !n->h_io[q]) NET_TRY(n, cudaMallocHost((void**)&n->h_io[q], (size_t)n->chunk * wbytes));
    }
    // Host runs with copies: a short first chunk (its input copy cannot overlap
    // compute) and a short last chunk (nor can its raster copy), chunk / 8
    // steps each, so the pipeline fills and drains quickly.
    const bool edges = host && (forced || raster) && steps >= 2 * (int64_t)n->chunk;
    const int64_t edge = std::max<int64_t>(1, n->chunk / 8);
    const int flags = (forced ? 1 : 0) | (current ? 2 : 0) | (raster ? 4 : 0);
    // the chunk plan, and every graph it needs captured and instantiated
    // before the run's first event: graph building never falls inside the
    // device time the run reports
    std::vector<std::pair<int, cudaGraphExec_t>> plan;
    for (int64_t done = 0, k = 0; done < steps; ++k) {
        const int64_t left = steps - done;
        int len = (int)std::min<int64_t>(n->chunk, left);
        if (edges) {
            if (k == 0 || left <= edge) len = (int)std::min<int64_t>(edge, left);
            else if (left < n->chunk + edge) len = (int)(left - edge);
        }
        cudaGraphExec_t ex = nullptr;
        if (!n->resident) {
            int rc = net_graph(n, len, flags, (int)(k & 1), (int)((n->steps_done + done) & 1), &ex);
            if (rc) return rc;
        }
        plan.emplace_back(len, ex);
        done += len;
    }
    size_t res_smem = 0;
    int res_nst = 0;
    if (n->resident) {  // checked before the run's first event, as the graphs are built
        std::string why;
        if (!res_check(n, &why, &res_smem, &res_nst)) return szsnn_set_error(n->ctx, SZSNN_ERR_STATE, why);
    }
    NET_TRY(n, cudaEventRecord(n->ev_run0, st));
    NET_TRY(n, cudaStreamWaitEvent(cp, n->ev_run0, 0));  // copies follow earlier work on the main stream
    NET_TRY(n, cudaStreamWaitEvent(cpo, n->ev_run0, 0));
    const cudaMemcpyKind in_kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind out_kind = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    struct Pending { bool on; size_t off, bytes; };
    Pending pend[2] = {{false, 0, 0}, {false, 0, 0}};
    auto flush = [&](int b) -> int {  // pageable copy-out of the chunk held in bounce buffer b
        if (!pend[b].on) return SZSNN_OK;
        NET_TRY(n, cudaEventSynchronize(n->ev_out[b]));
        std::memcpy((char*)raster + pend[b].off, n->h_io[2 + b], pend[b].bytes);
        pend[b].on = false;
        return SZSNN_OK;
    };
    int64_t done = 0;
    for (size_t k = 0; k < plan.size(); ++k) {
        const int b = (int)(k & 1);
        const int len = plan[k].first;
        const size_t bytes = (size_t)len * wbytes, off = (size_t)done * wbytes;
        if (forced) {
            if (k >= 2) NET_TRY(n, cudaStreamWaitEvent(cp, n->ev_comp[b], 0));  // stage b read by chunk k-2
            const char* src = (const char*)forced + off;
            if (bounce_in) {
                if (k >= 2) NET_TRY(n, cudaEventSynchronize(n->ev_in[b]));  // bounce b copied for chunk k-2
                std::memcpy(n->h_io[b], src, bytes);
                src = (const char*)n->h_io[b];
            }
            NET_TRY(n, cudaMemcpyAsync(n->d_forced_stage[b], src, bytes, in_kind, cp));
            NET_TRY(n, cudaEventRecord(n->ev_in[b], cp));
            NET_TRY(n, cudaStreamWaitEvent(st, n->ev_in[b], 0));
        }
        if (current && n->N)
            NET_TRY(n, cudaMemcpyAsync(n->d_current_stage, current + (size_t)done * n->N, (size_t)len * n->N * 4, in_kind, st));
        if (raster && k >= 2) NET_TRY(n, cudaStreamWaitEvent(st, n->ev_out[b], 0));  // stage b copied out
        if (n->resident) {
            NET_TRY(n, launch_resident(n, len, flags, b, st, res_smem, res_nst));
            n->kernel_launches += 1;
        } else {
            NET_TRY(n, cudaGraphLaunch(plan[k].second, st));
            n->graph_launches += 1;
            n->kernel_launches += (uint64_t)((n->overlap ? 1 : 2) + (n->mon_n ? 1 : 0)) * len + 1;
        }
        NET_TRY(n, cudaEventRecord(n->ev_comp[b], st));
        if (raster) {
            int rc = flush(b);  // bounce b last held chunk k-2
            if (rc) return rc;
            NET_TRY(n, cudaStreamWaitEvent(cpo, n->ev_comp[b], 0));
            char* dst = bounce_out ? (char*)n->h_io[2 + b] : (char*)raster + off;
            NET_TRY(n, cudaMemcpyAsync(dst, n->d_raster_stage[b], bytes, out_kind, cpo));
            NET_TRY(n, cudaEventRecord(n->ev_out[b], cpo));
            if (bounce_out) pend[b] = Pending{true, off, bytes};
            rc = flush(b ^ 1);  // chunk k-1, copied while chunk k computes
            if (rc) return rc;
        }
        done += len;
    }
    n->steps_done += steps;
    for (int b = 0; b < 2; ++b) {
        int rc = flush(b);
        if (rc) return rc;
    }
    // the main stream resumes after the last copies of both directions
    NET_TRY(n, cudaEventRecord(n->ev_in[0], cp));
    NET_TRY(n, cudaStreamWaitEvent(st, n->ev_in[0], 0));
    NET_TRY(n, cudaEventRecord(n->ev_out[0], cpo));
    NET_TRY(n, cudaStreamWaitEvent(st, n->ev_out[0], 0));
    NET_TRY(n, cudaEventRecord(n->ev_run1, st));
    n->run_timed = true;
    if (host) NET_TRY(n, cudaStreamSynchronize(st));  // host arrays are complete on return
    return SZSNN_OK;
}

extern "C" int szsnn_net_run(szsnn_net* n, int64_t steps, const uint32_t* forced_host, uint32_t* raster_host)
{
    return net_run_impl(n, steps, forced_host, nullptr, raster_host, true);
}

extern "C" int szsnn_net_run_device(szsnn_net* n, int64_t steps, const uint32_t* forced_dev, const float* current_dev,
                                    uint32_t* raster_dev)
{
    return net_run_impl(n, steps, forced_dev, current_dev, raster_dev, false);
}

// Per-kernel device time.  The network's state, inputs, ring counters and
// statistics are copied to scratch buffers; a CUDA graph then replays
// `steps` delivery launches, `steps` update launches and `steps` whole steps
// of the current step (the clock does not advance, so every replay repeats the
// same work: the delivery reads ring slots of past steps, the update re-fills
// slot t of the scratch counters and ids of a slot that no live delivery
// reads).  Events bracket each group of launches on the launching stream; the
// real network is left untouched.  Overlapped order: the delivery timed alone
// is far(t+1) (delays >= 2), the update includes its m = 1 deliveries, and the
// whole step is the fused k_step.
static int net_profile_impl(szsnn_net* n, int64_t steps, double* prop_ms, double* upd_ms, double* step_ms,
                            double* events_per_launch)
{
    if (!n || steps < 1 || steps > 100000) return SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream;
    const size_t U = (size_t)n->U, N = (size_t)std::max<int64_t>(n->N, 1);
    NetDev d = make_dev(n);
    float* sst[4] = {};
    float* sin[4] = {};        // e0, i0, e1, i1
    long long* sfx[4] = {};
    uint32_t* scnt = nullptr;
    unsigned long long* sstats = nullptr;  // [0..3] live, [4..7] copy after the delivery replays
    cudaEvent_t ev[4] = {};
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaSuccess;
    auto fin = [&](cudaError_t err) {
        if (ex) cudaGraphExecDestroy(ex);
        if (g) cudaGraphDestroy(g);
        for (auto& x : ev) if (x) cudaEventDestroy(x);
        for (auto& x : sst) cudaFree(x);
        for (auto& x : sin) cudaFree(x);
        for (auto& x : sfx) cudaFree(x);
        cudaFree(scnt); cudaFree(sstats);
        return err;
    };
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
        e = dalloc(&sst[k], U);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sst[k], n->d_st[k], U * 4, cudaMemcpyDeviceToDevice, st);
    }
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
        const float* src = (k & 1) ? n->d_in_i[k >> 1] : n->d_in_e[k >> 1];
        e = dalloc(&sin[k], N);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sin[k], src, N * 4, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && n->acc_mode == SZSNN_ACC_FIXED) {
            e = dalloc(&sfx[k], N);
            if (e == cudaSuccess) e = cudaMemsetAsync(sfx[k], 0, N * 8, st);
        }
    }
    if (e == cudaSuccess) e = dalloc(&scnt, (size_t)n->R);
    if (e == cudaSuccess) e = cudaMemcpyAsync(scnt, n->d_ring_cnt, (size_t)n->R * 4, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = dalloc(&sstats, 8);
    if (e == cudaSuccess) e = cudaMemsetAsync(sstats, 0, 64, st);
    for (auto& x : ev) if (e == cudaSuccess) e = cudaEventCreate(&x);
    if (e != cudaSuccess) return szsnn_set_error(n->ctx, SZSNN_ERR_CUDA, std::string("profile: ") + cudaGetErrorString(fin(e)));
    d.st0 = sst[0]; d.st1 = sst[1]; d.st2 = sst[2]; d.st3 = sst[3];
    d.in_e = sin[0]; d.in_i = sin[1]; d.in_e1 = sin[2]; d.in_i1 = sin[3];
    d.fx_e = sfx[0]; d.fx_i = sfx[1]; d.fx_e1 = sfx[2]; d.fx_i1 = sfx[3];
    d.ring_cnt = scnt; d.stats = sstats; d.group = nullptr; d.group_spikes = nullptr;
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(ev[0], st, cudaEventRecordExternal);
    for (int64_t k = 0; k < steps && e == cudaSuccess; ++k)
        e = n->overlap ? launch_propagate_far(n, d, 1, st) : launch_propagate_classic(n, d, 0, st);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(ev[1], st, cudaEventRecordExternal);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sstats + 4, sstats, 32, cudaMemcpyDeviceToDevice, st);
    // each update replay re-fills slot t from empty (a replay adds the step's
    // spikes again; without the reset a busy network would overflow the slot)
    uint32_t* slot_t = scnt + (size_t)(n->steps_done % n->R);
    for (int64_t k = 0; k < steps && e == cudaSuccess; ++k) {
        e = cudaMemsetAsync(slot_t, 0, 4, st);
        if (e == cudaSuccess) e = launch_update(n, d, 0, nullptr, nullptr, nullptr, st);
    }
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(ev[2], st, cudaEventRecordExternal);
    for (int64_t k = 0; k < steps && e == cudaSuccess; ++k) {
        if (n->overlap) {
            e = cudaMemsetAsync(slot_t, 0, 4, st);
            if (e == cudaSuccess) e = launch_step(n, d, 0, nullptr, nullptr, nullptr, st);
        } else {  // classic propagate empties slot t itself
            e = launch_propagate_classic(n, d, 0, st);
            if (e == cudaSuccess) e = launch_update(n, d, 0, nullptr, nullptr, nullptr, st);
        }
    }
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(ev[3], st, cudaEventRecordExternal);
    cudaError_t e2 = cudaStreamEndCapture(st, &g);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(ex, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float a = 0, b = 0, c = 0;
    unsigned long long hs[8] = {};
    if (e == cudaSuccess) e = cudaEventElapsedTime(&a, ev[0], ev[1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&b, ev[1], ev[2]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&c, ev[2], ev[3]);
    if (e == cudaSuccess) e = cudaMemcpy(hs, sstats, sizeof(hs), cudaMemcpyDeviceToHost);
    fin(cudaSuccess);
    if (e != cudaSuccess) return szsnn_set_error(n->ctx, SZSNN_ERR_CUDA, std::string("profile: ") + cudaGetErrorString(e));
    n->t_prop_ms = a;
    n->t_upd_ms = b;
    if (prop_ms) *prop_ms = a;
    if (upd_ms) *upd_ms = b;
    if (step_ms) *step_ms = c;
    if (events_per_launch) *events_per_launch = (double)(hs[4] + hs[6] + hs[7]) / (double)steps;
    return SZSNN_OK;
}

extern "C" int szsnn_net_profile(szsnn_net* n, int64_t steps, double* prop_ms, double* upd_ms, double* events_per_launch)
{
    return net_profile_impl(n, steps, prop_ms, upd_ms, nullptr, events_per_launch);
}

extern "C" int szsnn_net_profile_step(szsnn_net* n, int64_t steps, double* prop_ms, double* upd_ms, double* step_ms,
                                      double* events_per_launch)
{
    return net_profile_impl(n, steps, prop_ms, upd_ms, step_ms, events_per_launch);
}

extern "C" int szsnn_net_timing(szsnn_net* n, double* prop_ms, double* upd_ms, double* total_ms)
{
    if (!n) return SZSNN_ERR_ARG;
    if (n->run_timed) {  // device time of the last szsnn_net_run / szsnn_net_run_device
        NET_TRY(n, cudaEventSynchronize(n->ev_run1));
        float ms = 0;
        NET_TRY(n, cudaEventElapsedTime(&ms, n->ev_run0, n->ev_run1));
        n->t_total_ms = ms;
    }
    if (prop_ms) *prop_ms = n->t_prop_ms;
    if (upd_ms) *upd_ms = n->t_upd_ms;
    if (total_ms) *total_ms = n->t_total_ms;
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_tuning(szsnn_net* n, int mode, int group, int blocks, int upd_block)
{
    if (!n) return SZSNN_ERR_ARG;
    if (mode != 0 && mode != 1) return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "propagate mode must be 0 or 1");
    if (mode == 0 && group != 0 && group != 4 && group != 8 && group != 16 && group != 32)
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "grouped propagate: lanes per bucket must be 4, 8, 16 or 32");
    if (mode == 1 && group != 0 && group != 8 && group != 16 && group != 32)
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "flattened propagate: items per warp must be 8, 16 or 32");
    if (upd_block != 0 && (upd_block < 32 || upd_block > UPD_MAX_BLOCK || upd_block % 32))
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "update block must be a multiple of 32 in 32..256");
    n->prop_mode = mode;
    n->prop_group = group ? group : (mode == 1 ? 32 : 16);
    if (blocks >= 0) n->prop_blocks = blocks;
    if (upd_block) n->upd_block = upd_block;
    NET_TRY(n, fill_blk_pop(n));
    for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);
    n->graphs.clear();
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_update_units(szsnn_net* n, int units_per_thread)
{
    if (!n) return SZSNN_ERR_ARG;
    if (units_per_thread < 0 || units_per_thread > UPD_MAX_UPT)
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "units per update thread must be in 0..16 (0: automatic)");
    const int old = n->upd_units;
    n->upd_units = units_per_thread;
    // a block tile must fit the shared memory of one block
    const size_t bytes = tile_smem_bytes((int64_t)upd_upt(n) * n->upd_block, n->acc_mode == SZSNN_ACC_FIXED);
    if (bytes > 200 * 1024) {
        n->upd_units = old;
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "the update block's tile exceeds shared memory");
    }
    NET_TRY(n, fill_blk_pop(n));
    for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);
    n->graphs.clear();
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_update_tiles(szsnn_net* n, int mode, int blocks_per_sm)
{
    if (!n) return SZSNN_ERR_ARG;
    if (mode < 0 || mode > 2) return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "update tile mode must be 0, 1 or 2");
    if (blocks_per_sm < 0 || blocks_per_sm > 32)
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "update blocks per SM must be in 0..32");
    n->upd_tiles = mode;
    n->upd_per_sm = blocks_per_sm;
    for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);
    n->graphs.clear();
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_resident(szsnn_net* n, int on, int update_warps, int blocks)
{
    if (!n) return SZSNN_ERR_ARG;
    if (on != 0 && on != 1) return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "resident must be 0 or 1");
    if (update_warps < 0 || update_warps > RES_THREADS / 32 - 1)
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "update warps must be in 0..31 (0: 16)");
    if (blocks < 0 || blocks > 4096) return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "blocks must be in 0..4096");
    const bool was = n->resident;
    const int uw0 = n->res_uw, nb0 = n->res_blocks;
    n->resident = on != 0;
    n->res_uw = update_warps > 0 ? update_warps : 16;
    n->res_blocks = blocks;
    if (n->resident) {
        std::string why;
        size_t smem = 0;
        int nst = 0;
        if (!res_check(n, &why, &smem, &nst)) {
            n->resident = was;
            n->res_uw = uw0;
            n->res_blocks = nb0;
            return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, why);
        }
    }
    return SZSNN_OK;
}

extern "C" int szsnn_net_stats_get(szsnn_net* n, szsnn_net_stats* out)
{
    if (!n || !out) return SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream;
    unsigned long long s[4] = {0, 0, 0, 0};
    long long clock = 0;
    uint32_t newest = 0;
    NET_TRY(n, cudaMemcpyAsync(s, n->d_stats, sizeof(s), cudaMemcpyDeviceToHost, st));
    NET_TRY(n, cudaMemcpyAsync(&clock, n->d_clock, 8, cudaMemcpyDeviceToHost, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    if (clock >= 1) {
        NET_TRY(n, cudaMemcpyAsync(&newest, n->d_ring_cnt + ((clock - 1) % n->R), 4, cudaMemcpyDeviceToHost, st));
        NET_TRY(n, cudaStreamSynchronize(st));
    }
    out->steps_done = clock;
    out->events = s[0];
    out->spikes = s[1] + newest;
    out->graph_launches = n->graph_launches;
    out->kernel_launches = n->kernel_launches;
    return SZSNN_OK;
}

extern "C" int szsnn_net_group_spikes(szsnn_net* n, uint64_t* counts, int reset)
{
    if (!n || !counts || !n->d_group_spikes) return n ? szsnn_set_error(n->ctx, SZSNN_ERR_STATE, "network has no groups") : SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream;
    NET_TRY(n, cudaMemcpyAsync(counts, n->d_group_spikes, (size_t)n->n_groups * 8, cudaMemcpyDeviceToHost, st));
    if (reset) NET_TRY(n, cudaMemsetAsync(n->d_group_spikes, 0, (size_t)n->n_groups * 8, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    return SZSNN_OK;
}

extern "C" int szsnn_net_get_state(szsnn_net* n, int slot, float* host)
{
    if (!n || slot < 0 || slot > 3 || !host) return SZSNN_ERR_ARG;
    NET_TRY(n, cudaMemcpyAsync(host, n->d_st[slot], (size_t)n->U * 4, cudaMemcpyDeviceToHost, n->ctx->stream));
    NET_TRY(n, cudaStreamSynchronize(n->ctx->stream));
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_monitor(szsnn_net* n, const int32_t* ids, int32_t n_ids, uint32_t slot_mask,
                                     int64_t capacity)
{
    if (!n) return SZSNN_ERR_ARG;
    if (n_ids < 0 || (n_ids > 0 && (!ids || slot_mask == 0 || slot_mask > 15u || capacity < 1)))
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG,
                               "szsnn_net_set_monitor: ids, a slot mask in 1..15 and a capacity >= 1 are needed");
    for (int32_t i = 0; i < n_ids; ++i)
        if (ids[i] < 0 || ids[i] >= n->U)
            return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "szsnn_net_set_monitor: unit id outside 0..U-1");
    cudaStream_t st = n->ctx->stream;
    NET_TRY(n, cudaStreamSynchronize(st));  // no step in flight writes the old trace
    cudaFree(n->d_mon_ids);
    cudaFree(n->d_mon_buf);
    n->d_mon_ids = nullptr;
    n->d_mon_buf = nullptr;
    n->mon_n = 0;
    n->mon_slots = 0;
    n->mon_cap = 0;
    for (auto& kv : n->graphs) cudaGraphExecDestroy(kv.second);  // graphs hold the monitor launches or not
    n->graphs.clear();
    if (n_ids == 0) return SZSNN_OK;
    const size_t ns = (size_t)__builtin_popcount(slot_mask);
    NET_TRY(n, dalloc(&n->d_mon_ids, (size_t)n_ids));
    NET_TRY(n, dalloc(&n->d_mon_buf, (size_t)capacity * ns * (size_t)n_ids));
    if (!n->d_mon_t0) NET_TRY(n, dalloc(&n->d_mon_t0, 1));
    n->mon_t0 = n->steps_done;
    NET_TRY(n, cudaMemcpyAsync(n->d_mon_ids, ids, (size_t)n_ids * 4, cudaMemcpyHostToDevice, st));
    NET_TRY(n, cudaMemcpyAsync(n->d_mon_t0, &n->mon_t0, 8, cudaMemcpyHostToDevice, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    n->mon_n = n_ids;
    n->mon_slots = slot_mask;
    n->mon_cap = capacity;
    return SZSNN_OK;
}

extern "C" int szsnn_net_monitor_read(szsnn_net* n, float* out, int64_t max_steps, int64_t* steps_out,
                                      int64_t* dropped_out)
{
    if (!n || max_steps < 0 || (max_steps > 0 && !out)) return SZSNN_ERR_ARG;
    if (!n->mon_n) return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "szsnn_net_monitor_read: no monitor is set");
    cudaStream_t st = n->ctx->stream;
    const int64_t recorded = n->steps_done - n->mon_t0;
    const int64_t kept = std::min<int64_t>(recorded, n->mon_cap);
    const int64_t steps = std::min<int64_t>(kept, max_steps);
    const size_t row = (size_t)__builtin_popcount(n->mon_slots) * (size_t)n->mon_n;
    if (steps > 0) NET_TRY(n, cudaMemcpyAsync(out, n->d_mon_buf, (size_t)steps * row * 4, cudaMemcpyDeviceToHost, st));
    n->mon_t0 = n->steps_done;  // recording restarts at the current step
    NET_TRY(n, cudaMemcpyAsync(n->d_mon_t0, &n->mon_t0, 8, cudaMemcpyHostToDevice, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    if (steps_out) *steps_out = steps;
    if (dropped_out) *dropped_out = recorded - steps;
    return SZSNN_OK;
}

extern "C" int szsnn_net_set_state(szsnn_net* n, int slot, const float* host)
{
    if (!n || slot < 0 || slot > 3 || !host) return SZSNN_ERR_ARG;
    NET_TRY(n, cudaMemcpyAsync(n->d_st[slot], host, (size_t)n->U * 4, cudaMemcpyHostToDevice, n->ctx->stream));
    NET_TRY(n, cudaStreamSynchronize(n->ctx->stream));
    return SZSNN_OK;
}

// checkpoint blob: header | 4 state slots | ring counts | ring ids | stats
struct CkptHeader { uint64_t magic, U, D, clock; };
static const uint64_t kCkptMagic = 0x535A534E4E434B31ull;  // "SZSNNCK1"

extern "C" int szsnn_net_checkpoint_size(szsnn_net* n, uint64_t* bytes)
{
    if (!n || !bytes) return SZSNN_ERR_ARG;
    *bytes = sizeof(CkptHeader) + (uint64_t)4 * n->U * 4 + (uint64_t)n->R * 4 + (uint64_t)n->R * n->U * 4 + 32;
    return SZSNN_OK;
}

extern "C" int szsnn_net_checkpoint(szsnn_net* n, void* blob, uint64_t bytes)
{
    uint64_t need = 0;
    if (szsnn_net_checkpoint_size(n, &need) || !blob || bytes < need) return n ? szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "checkpoint buffer too small") : SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream;
    char* p = (char*)blob;
    CkptHeader h{kCkptMagic, (uint64_t)n->U, (uint64_t)n->D, 0};
    NET_TRY(n, cudaMemcpyAsync(&h.clock, n->d_clock, 8, cudaMemcpyDeviceToHost, st));
    char* q = p + sizeof(CkptHeader);
    for (int k = 0; k < 4; ++k) {
        NET_TRY(n, cudaMemcpyAsync(q, n->d_st[k], (size_t)n->U * 4, cudaMemcpyDeviceToHost, st));
        q += (size_t)n->U * 4;
    }
    NET_TRY(n, cudaMemcpyAsync(q, n->d_ring_cnt, (size_t)n->R * 4, cudaMemcpyDeviceToHost, st));
    q += (size_t)n->R * 4;
    NET_TRY(n, cudaMemcpyAsync(q, n->d_ring_ids, (size_t)n->R * n->U * 4, cudaMemcpyDeviceToHost, st));
    q += (size_t)n->R * n->U * 4;
    NET_TRY(n, cudaMemcpyAsync(q, n->d_stats, 32, cudaMemcpyDeviceToHost, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    std::memcpy(p, &h, sizeof(h));
    return SZSNN_OK;
}

extern "C" int szsnn_net_restore(szsnn_net* n, const void* blob, uint64_t bytes)
{
    uint64_t need = 0;
    if (szsnn_net_checkpoint_size(n, &need) || !blob || bytes < need) return n ? szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "checkpoint blob too small") : SZSNN_ERR_ARG;
    const char* p = (const char*)blob;
    CkptHeader h;
    std::memcpy(&h, p, sizeof(h));
    if (h.magic != kCkptMagic || h.U != (uint64_t)n->U || h.D != (uint64_t)n->D)
        return szsnn_set_error(n->ctx, SZSNN_ERR_ARG, "checkpoint does not match this network");
    cudaStream_t st = n->ctx->stream;
    const char* q = p + sizeof(CkptHeader);
    for (int k = 0; k < 4; ++k) {
        NET_TRY(n, cudaMemcpyAsync(n->d_st[k], q, (size_t)n->U * 4, cudaMemcpyHostToDevice, st));
        q += (size_t)n->U * 4;
    }
    NET_TRY(n, cudaMemcpyAsync(n->d_ring_cnt, q, (size_t)n->R * 4, cudaMemcpyHostToDevice, st));
    q += (size_t)n->R * 4;
    NET_TRY(n, cudaMemcpyAsync(n->d_ring_ids, q, (size_t)n->R * n->U * 4, cudaMemcpyHostToDevice, st));
    q += (size_t)n->R * n->U * 4;
    NET_TRY(n, cudaMemcpyAsync(n->d_stats, q, 32, cudaMemcpyHostToDevice, st));
    long long clock = (long long)h.clock;
    NET_TRY(n, cudaMemcpyAsync(n->d_clock, &clock, 8, cudaMemcpyHostToDevice, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    n->steps_done = clock;
    if (n->mon_n) {  // the monitor's trace restarts at the restored step
        n->mon_t0 = clock;
        NET_TRY(n, cudaMemcpyAsync(n->d_mon_t0, &n->mon_t0, 8, cudaMemcpyHostToDevice, st));
        NET_TRY(n, cudaStreamSynchronize(st));
    }
    return net_prime(n);
}

extern "C" int szsnn_net_get_synapses(szsnn_net* n, uint64_t* row_ptr, int32_t* tgt, float* w)
{
    if (!n) return SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream;
    if (row_ptr)
        NET_TRY(n, cudaMemcpyAsync(row_ptr, n->d_row_ptr, ((size_t)n->U * n->D + 1) * 8, cudaMemcpyDeviceToHost, st));
    if ((tgt || w) && n->n_syn) {
        int32_t* dt = nullptr;
        float* dw = nullptr;
        NET_TRY(n, dalloc(&dt, (size_t)n->n_syn));
        NET_TRY(n, dalloc(&dw, (size_t)n->n_syn));
        k_unpack_syn<<<1024, 256, 0, st>>>(n->d_syn, dt, dw, n->n_syn);
        NET_TRY(n, cudaGetLastError());
        if (tgt) NET_TRY(n, cudaMemcpyAsync(tgt, dt, (size_t)n->n_syn * 4, cudaMemcpyDeviceToHost, st));
        if (w) NET_TRY(n, cudaMemcpyAsync(w, dw, (size_t)n->n_syn * 4, cudaMemcpyDeviceToHost, st));
        NET_TRY(n, cudaStreamSynchronize(st));
        cudaFree(dt);
        cudaFree(dw);
    }
    NET_TRY(n, cudaStreamSynchronize(st));
    return SZSNN_OK;
}

extern "C" int szsnn_net_check_finite(szsnn_net* n, int* finite_out)
{
    if (!n || !finite_out) return SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream;
    uint32_t* flag = nullptr;
    NET_TRY(n, dalloc(&flag, 1));
    NET_TRY(n, cudaMemsetAsync(flag, 0, 4, st));
    for (int k = 0; k < 4; ++k) {
        k_check_finite<<<512, 256, 0, st>>>(n->d_st[k], n->U, flag);
        NET_TRY(n, cudaGetLastError());
    }
    uint32_t h = 0;
    NET_TRY(n, cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    cudaFree(flag);
    *finite_out = h ? 0 : 1;
    if (h) {
        uint32_t code = SZSNN_DEV_NONFINITE, zero = 0;
        // record as the sticky device error when none is set yet
        uint32_t cur[2] = {0, 0};
        NET_TRY(n, cudaMemcpy(cur, n->ctx->d_err, 8, cudaMemcpyDeviceToHost));
        if (cur[0] == 0) {
            NET_TRY(n, cudaMemcpy(n->ctx->d_err, &code, 4, cudaMemcpyHostToDevice));
            NET_TRY(n, cudaMemcpy(n->ctx->d_err + 1, &zero, 4, cudaMemcpyHostToDevice));
        }
    }
    return SZSNN_OK;
}

extern "C" int szsnn_net_last_inputs(szsnn_net* n, float* in_exc, float* in_inh)
{
    if (!n) return SZSNN_ERR_ARG;
    cudaStream_t st = n->ctx->stream;
    if (in_exc && n->N) NET_TRY(n, cudaMemcpyAsync(in_exc, n->d_dbg_in, (size_t)n->N * 4, cudaMemcpyDeviceToHost, st));
    if (in_inh && n->N)
        NET_TRY(n, cudaMemcpyAsync(in_inh, n->d_dbg_in + std::max<int64_t>(n->N, 1), (size_t)n->N * 4, cudaMemcpyDeviceToHost, st));
    NET_TRY(n, cudaStreamSynchronize(st));
    return SZSNN_OK;
}

// ---------------------------------------------------------------------------
// szsnn_step_static: one step that allocates nothing.
//
// For callers that cannot call cudaMalloc: hosts that own and partition all
// device memory themselves (a fixed-budget pool or arena, a framework's
// caching allocator) and forbid libraries from allocating, and real-time
// step loops that cannot afford cudaMalloc's implicit device synchronisation
// and unbounded latency.  The caller passes every input and output buffer;
// the step's scratch -- the per-step input accumulators plus a small header
// (step counter, statistics, population table, error word) -- lives in the
// file-scope array below, which every GPU that loads this library holds until
// the process exits.
//
// Limits and sharing: at most SZSNN_STATIC_MAX_NEURONS neurons (larger
// networks are rejected with SZSNN_ERR_LIMIT).  All calls on a device share
// the one array and it keeps the last call's contents; each call clears the
// parts that must start at zero before it launches.  Calls whose work
// overlaps on the GPU (different streams, or threads launching at once)
// race on the array and must be serialised by the caller.
// ---------------------------------------------------------------------------
#define SZSNN_STATIC_HDR_BYTES 4096
static __device__ __align__(256) unsigned char
    g_static_scratch[SZSNN_STATIC_HDR_BYTES + 2 * sizeof(float) * SZSNN_STATIC_MAX_NEURONS];

// Header of one call, written by a kernel whose parameters carry the
// population table and the step number by value (nothing is read from host
// memory after the call returns): [0] step counter, [64] statistics zeroed,
// [256] population table.
__global__ void k_static_setup(PopDev p0, PopDev p1, long long clock, unsigned char* base)
{
    const int w = (int)(sizeof(PopDev) / 8);
    unsigned long long* tab = reinterpret_cast<unsigned long long*>(base + 256);
    const unsigned long long* a = reinterpret_cast<const unsigned long long*>(&p0);
    const unsigned long long* b = reinterpret_cast<const unsigned long long*>(&p1);
    for (int i = threadIdx.x; i < 2 * w; i += blockDim.x) tab[i] = i < w ? a[i] : b[i - w];
    if (threadIdx.x < 8) reinterpret_cast<unsigned long long*>(base + 64)[threadIdx.x] = 0ull;
    if (threadIdx.x == 0) *reinterpret_cast<long long*>(base) = clock;
}

#include <mutex>

namespace {
std::mutex g_static_mu;
void* g_static_addr[64] = {};  // device address of g_static_scratch per device
int g_static_sms[64] = {};

int static_fail(char* err, size_t len, int code, const std::string& m)
{
    if (err && len) {
        std::strncpy(err, m.c_str(), len - 1);
        err[len - 1] = 0;
    }
    return code;
}
}  // namespace

extern "C" int szsnn_step_static(const szsnn_static_step* s, char* err, size_t err_len)
{
    if (!s) return static_fail(err, err_len, SZSNN_ERR_ARG, "szsnn_step_static: null argument");
    const int64_t N = s->n_neurons, P = s->n_sources, U = N + P;
    const int D = s->max_delay;
    if (N < 1 || P < 0 || D < 1 || D > 1024 || s->step < 0)
        return static_fail(err, err_len, SZSNN_ERR_ARG, "szsnn_step_static: bad sizes or step");
    if (N > SZSNN_STATIC_MAX_NEURONS)
        return static_fail(err, err_len, SZSNN_ERR_LIMIT,
                           "szsnn_step_static: " + std::to_string(N) + " neurons exceed the static scratch maximum of " +
                               std::to_string(SZSNN_STATIC_MAX_NEURONS));
    if (U > 0x7fffffffLL)
        return static_fail(err, err_len, SZSNN_ERR_LIMIT, "szsnn_step_static: more than 2^31-1 units");
    if (s->model != SZSNN_IF_CURR_EXP && s->model != SZSNN_IF_COND_EXP && s->model != SZSNN_IZHIKEVICH)
        return static_fail(err, err_len, SZSNN_ERR_ARG, "szsnn_step_static: model must be a neuron model");
    if (!s->row_ptr || (!s->syn && U > 0) || !s->state[0] || !s->state[1] || !s->state[2] || !s->state[3] ||
        !s->ring_cnt || !s->ring_ids)
        return static_fail(err, err_len, SZSNN_ERR_ARG, "szsnn_step_static: null device buffer");
    if (!s->error_word)
        return static_fail(err, err_len, SZSNN_ERR_ARG,
                           "szsnn_step_static: error_word is required (device errors are reported there)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return static_fail(err, err_len, SZSNN_ERR_CUDA, std::string("szsnn_step_static: cudaGetDevice: ") + cudaGetErrorString(e));
    unsigned char* base = nullptr;
    int sms = 148;
    {
        // once per device, with that device current: the device address of the
        // static array (the host-side symbol is only a stand-in for it)
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!g_static_addr[dev]) {
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_static_scratch);
            if (e != cudaSuccess || !ptr)
                return static_fail(err, err_len, SZSNN_ERR_CUDA,
                                   std::string("szsnn_step_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            int v = 148;
            if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) v = 148;
            g_static_sms[dev] = v;
            g_static_addr[dev] = ptr;
        }
        base = (unsigned char*)g_static_addr[dev];
        sms = g_static_sms[dev];
    }
    cudaStream_t st = (cudaStream_t)s->stream;
    // header layout: [0] step counter, [64] statistics, [256] population table
    PopDev hp[2];
    std::memset(hp, 0, sizeof(hp));
    hp[0].model = s->model; hp[0].flags = s->flags; hp[0].begin = 0; hp[0].end = N;
    std::memcpy(hp[0].p, s->params, sizeof(s->params));
    if (s->model != SZSNN_IZHIKEVICH) { hp[0].p[12] = sz_decay(s->params[4]); hp[0].p[13] = sz_decay(s->params[5]); }
    hp[1].model = SZSNN_POISSON; hp[1].begin = N; hp[1].end = U; hp[1].p[0] = s->source_p; hp[1].seed = s->seed;
    float* acc = (float*)(base + SZSNN_STATIC_HDR_BYTES);
    k_static_setup<<<1, 64, 0, st>>>(hp[0], hp[1], (long long)s->step, base);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, 2 * sizeof(float) * (size_t)N, st);  // input accumulators
    if (e != cudaSuccess)
        return static_fail(err, err_len, SZSNN_ERR_CUDA, std::string("szsnn_step_static: set-up: ") + cudaGetErrorString(e));
    NetDev d{};
    d.N = N; d.U = U; d.words = sz_div_up(U, 32); d.D = D; d.npops = P > 0 ? 2 : 1;
    d.pops = (const PopDev*)(base + 256);
    d.row_ptr = (const unsigned long long*)s->row_ptr;
    d.syn = (const int2*)s->syn;
    d.st0 = s->state[0]; d.st1 = s->state[1]; d.st2 = s->state[2]; d.st3 = s->state[3];
    d.in_e = acc; d.in_i = acc + N;
    d.acc_mode = SZSNN_ACC_FLOAT;
    d.ring_cnt = s->ring_cnt; d.ring_ids = s->ring_ids;
    d.clock = (const long long*)base;
    d.stats = (unsigned long long*)(base + 64);
    d.err = s->error_word;
    d.upt = 1;
    d.own_lo[0] = 0; d.own_hi[0] = N;  // every unit is updated here
    d.own_lo[1] = N; d.own_hi[1] = U;
    k_propagate<16><<<sms * 16, 256, 0, st>>>(d, 0, 1, PF_ZERO_SLOT | PF_SPIKES);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        k_update<0><<<(unsigned)sz_div_up(U, 256), 256, 0, st>>>(d, 0, nullptr, nullptr, s->fired_words);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return static_fail(err, err_len, SZSNN_ERR_CUDA, std::string("szsnn_step_static: launch: ") + cudaGetErrorString(e));
    return SZSNN_OK;
}
