/*
 * szsnn_cuda.h -- C ABI of the B200 (sm_100a) implementation of SZSNN's
 * clock-driven simulation step.
 *
 * The reference drives four OpenCL kernels through szsnn::Context
 * (szsnn1.1/src/Context.hpp:77-303): createKernel / setKernelArg /
 * enqueueKernel / createBuffer / writeBuffer / readBuffer and a single in-order
 * command queue.  This header replaces that seam: plain pointers and sizes,
 * one CUDA stream per context, every call returns a status code (0 = ok) and
 * szsnn_last_error() gives the message (the reference throws SzsnnException on
 * any CL status, szsnn1.1/src/utils.h:144-155).
 *
 * Ownership: device buffers returned by szsnn_alloc belong to the context
 * until szsnn_free; host memory always belongs to the caller and is not
 * retained after a call returns.  A context is not thread-safe: calls on one
 * context must be serialised (the reference uses one host thread and one
 * queue, szsnn1.1/src/Context.cpp:213).
 *
 * Three groups of entry points:
 *  1. context and buffers                       (Context / DataBuffer seam)
 *  2. drop-in kernels on the reference layout   (the four .cl kernels, same
 *     argument lists, device pointers)
 *  3. native network path (delay-bucketed CSR, device spike ring, Poisson
 *     sources, IF_cond_exp, CUDA graphs), batched sweeps and the
 *     IF_curr_exp adjoint used by the pyszsnn autograd function.
 */
#ifndef SZSNN_CUDA_H
#define SZSNN_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define SZSNN_OK            0
#define SZSNN_ERR_ARG       1   /* bad argument (null pointer, size, range)          */
#define SZSNN_ERR_CUDA      2   /* CUDA runtime error                               */
#define SZSNN_ERR_NOMEM     3   /* device or host allocation failed                 */
#define SZSNN_ERR_LIMIT     4   /* layout limit of the reference format exceeded     */
#define SZSNN_ERR_DEVICE    5   /* device-side check failed (overflow, bad index)    */
#define SZSNN_ERR_TIMEOUT   6   /* bounded device wait expired                      */
#define SZSNN_ERR_STATE     7   /* call not valid in the current state              */

/* device-side sticky error codes (szsnn_device_error) */
#define SZSNN_DEV_OK             0
#define SZSNN_DEV_BAD_TARGET     1  /* synapse target outside the partition / network */
#define SZSNN_DEV_QUEUE_OVERFLOW 2  /* global or local queue slot full                */
#define SZSNN_DEV_RING_OVERFLOW  3  /* native spike ring slot full                    */
#define SZSNN_DEV_NONFINITE      4  /* NaN/Inf found by szsnn_net_check_finite        */
#define SZSNN_DEV_BAD_DELAY      5  /* delay outside 1..max_delay                     */
#define SZSNN_DEV_STEP_PARITY    6  /* launch parity disagrees with the step counter  */
#define SZSNN_DEV_WAIT_TIMEOUT   7  /* a bounded wait for a bulk copy ran out         */

typedef struct szsnn_ctx szsnn_ctx;
typedef struct szsnn_net szsnn_net;
typedef struct szsnn_layout szsnn_layout;

/* Compile-time constants of the reference (szsnn1.1/src/locales.h:17-46),
 * which it prepends to every kernel source (Context.cpp:260-274).  Here they
 * are run-time values fixed at context creation. */
typedef struct {
    uint32_t max_partition_size;  /* MAX_PARTITION_SIZE (<= 1024, multiple of 32)   */
    uint32_t threads_per_group;   /* THREADS_PER_GROUP = MPS / NEURONS_PER_WI        */
    uint32_t warp_size;           /* WARP_SIZE == BUNDLE_SIZE (<= 32)                */
    uint32_t max_synaptic_delay;  /* MAX_SYNAPTIC_DELAY (<= 64: uint64 delay bitmap) */
} szsnn_layout_consts;

/* --------------------------------------------- 1. context and buffers --- */
/* Context::setup (Context.cpp:136-224): pick device, create the queue. */
int szsnn_ctx_create(int device, const szsnn_layout_consts* consts, szsnn_ctx** out);
int szsnn_ctx_destroy(szsnn_ctx* ctx);
const char* szsnn_last_error(const szsnn_ctx* ctx);
/* Use an external CUDA stream (cudaStream_t) instead of the context's own. */
int szsnn_set_stream(szsnn_ctx* ctx, void* cuda_stream);
void* szsnn_get_stream(szsnn_ctx* ctx);

/* Context::createBuffer (Context.cpp:398-417) */
int szsnn_alloc(szsnn_ctx* ctx, size_t bytes, void** dev_out);
int szsnn_free(szsnn_ctx* ctx, void* dev);
/* Context::writeBuffer / readBuffer with CL_TRUE (Context.cpp:421-505): blocking */
int szsnn_h2d(szsnn_ctx* ctx, void* dev, const void* host, size_t bytes);
int szsnn_d2h(szsnn_ctx* ctx, void* host, const void* dev, size_t bytes);
int szsnn_memset(szsnn_ctx* ctx, void* dev, int value, size_t bytes);
/* cl::Event::wait + CommandQueue::finish (Simulation.ipp:409-419); also
 * reports the device-side sticky error as SZSNN_ERR_DEVICE. */
int szsnn_sync(szsnn_ctx* ctx);
int szsnn_device_error(szsnn_ctx* ctx, uint32_t* code_out, uint32_t* info_out);
int szsnn_clear_device_error(szsnn_ctx* ctx);

/* Options that replace the reference's -D kernel flags (Simulation.ipp:13-38). */
#define SZSNN_OPT_OUTPUT_SPARSE_INPUT   1  /* input kernel stores sparse spikes
                                              (-DSZSNN_KERNEL_OUTPUT_SPIKES, off when
                                              SZSNN_NO_INPUT_TO_OUTPUT == 1, locales.h:64-68) */
#define SZSNN_OPT_FIRED_OUTPUT_PARTS    2  /* partitions held by firedOutput: dense
                                              spike words beyond it are not written
                                              (the reference writes past the end for the
                                              input partition, Const_rate_update_kernel.cl:238) */
#define SZSNN_OPT_IZH_HALF_STEPS        3  /* Izhikevich: two 0.5 ms half-steps for v */
int szsnn_set_option(szsnn_ctx* ctx, int option, int64_t value);

/* ------------------------------ 2. drop-in kernels, reference layout ----
 * Argument lists are those bound by Simulation::prep*Kernel
 * (Simulation.ipp:214-340); all pointers are device pointers.  The launch
 * covers the partitions the reference's NDRange covers: arg 1 partitions. */

/* IF_curr_exp_update (cl/IF_curr_exp_update_kernel.cl:100-120) */
int szsnn_update_if_curr_exp(szsnn_ctx* ctx, uint64_t cycle, uint32_t localPartitionCount,
                             const uint32_t* partitionSizes, const float* neuronParams,
                             float* neuronVars, uint32_t isInputCurrent, float* inputCurrent,
                             float* current, uint32_t isInputFiring, uint32_t* inputFired,
                             uint32_t* firedCount, uint32_t* fired, uint32_t* firedOutput,
                             uint32_t partitionOffset, uint32_t globalPartitionCount);
/* Izhikevich_update (cl/Izhikevich_update_kernel.cl:95-115) */
int szsnn_update_izhikevich(szsnn_ctx* ctx, uint64_t cycle, uint32_t localPartitionCount,
                            const uint32_t* partitionSizes, const float* neuronParams,
                            float* neuronVars, uint32_t isInputCurrent, float* inputCurrent,
                            float* current, uint32_t isInputFiring, uint32_t* inputFired,
                            uint32_t* firedCount, uint32_t* fired, uint32_t* firedOutput,
                            uint32_t partitionOffset, uint32_t globalPartitionCount);
/* Const_rate_update (cl/Const_rate_update_kernel.cl:91-111) */
int szsnn_update_const_rate(szsnn_ctx* ctx, uint64_t cycle, uint32_t localPartitionCount,
                            const uint32_t* partitionSizes, const float* neuronParams,
                            float* neuronVars, uint32_t isInputCurrent, float* inputCurrent,
                            float* current, uint32_t isInputFiring, uint32_t* inputFired,
                            uint32_t* firedCount, uint32_t* fired, uint32_t* firedOutput,
                            uint32_t partitionOffset, uint32_t globalPartitionCount);
/* gather (cl/gather_kernel.cl:67-77) */
int szsnn_gather(szsnn_ctx* ctx, uint64_t cycle, uint32_t partitionCount,
                 const uint32_t* partitionSizes, float* current, uint64_t gqPitch,
                 uint32_t* gqBundleCounter, uint32_t* gqBundles, const uint32_t* targets,
                 const float* weights);
/* scatter (cl/scatter_kernel.cl:68-83); groupPtrs / groupMatrix are uint2
 * arrays passed as uint32 pairs, lqEntries is a short2 array as int16 pairs. */
int szsnn_scatter(szsnn_ctx* ctx, uint64_t cycle, uint32_t partitionCount,
                  uint32_t* firedCount, uint32_t* fired, uint32_t groupPitch, uint32_t groupStep,
                  const uint32_t* groupPtrs, const uint32_t* groupMatrix, uint64_t gqPitch,
                  uint32_t* gqBundleCounter, uint32_t* gqBundles, uint32_t* lqEntryCounter,
                  int16_t* lqEntries, const uint64_t* delayBits);

/* Reference-layout builder (host only, no GPU needed): restates
 * NeuronData/SynapseData/SynapseIndex/GroupData/GlobalQueue/LocalQueue/
 * SpikeBuffer/CurrentData::initialize (NeuronData.ipp:27-170,
 * SynapseData.ipp:8-111, SynapseIndex.cpp:42-63, GroupData.cpp:70-228,
 * GlobalQueue.cpp:13-45, LocalQueue.cpp:32-70, SpikeBuffer.cpp:34-95,
 * CurrentData.ipp:15-50).  Synapse ids are global ids: neurons 0..N-1 and
 * inputs at Pn*MPS + i (NetworkGraph::connectInput, NetworkGraph.ipp:520-536).
 * delay1 is the stored delay (user delay + 1, NetworkGraph.ipp:431). */
typedef struct {
    uint32_t n_neurons;
    uint32_t n_inputs;
    uint32_t neuron_param_count, neuron_var_count;  /* model traits (neuron_model_traits.hpp) */
    uint32_t input_param_count, input_var_count;
    const float* neuron_params;   /* [n_neurons][param_count] row-major, or NULL */
    const float* neuron_vars;     /* [n_neurons][var_count]   */
    const float* input_params;    /* [n_inputs][input_param_count] */
    const float* input_vars;
    uint64_t n_synapses;
    const uint32_t* src;          /* global ids */
    const uint32_t* tgt;
    const float* weight;
    const uint32_t* delay1;
    uint32_t add_phony_synapse;   /* NetworkGraph::_addPhonySynapse (NetworkGraph.hpp:127-135) */
} szsnn_layout_desc;

/* array ids for szsnn_layout_array */
enum {
    SZSNN_L_PARTITION_SIZES = 0, /* uint32 [Ptot]                              */
    SZSNN_L_NEURON_PARAMS,       /* float  [pc][Pn][MPS]                       */
    SZSNN_L_NEURON_VARS,         /* float  [vc][Pn][MPS]                       */
    SZSNN_L_INPUT_PARAMS,        /* float  [ipc][1][MPS]                       */
    SZSNN_L_INPUT_VARS,          /* float  [ivc][1][MPS]                       */
    SZSNN_L_TARGETS,             /* uint32 [bundles][BUNDLE]                   */
    SZSNN_L_WEIGHTS,             /* float  [bundles][BUNDLE]                   */
    SZSNN_L_DELAY_BITS,          /* uint64 [network size]                      */
    SZSNN_L_GROUP_PTRS,          /* uint2  [Ptot][MPS][D]                      */
    SZSNN_L_GROUP_MATRIX,        /* uint2  [words allocated]                   */
    SZSNN_L_GQ_COUNTER,          /* uint32 [ALIGN(2*Ptot,32)]                  */
    SZSNN_L_GQ_BUNDLES,          /* uint32 [2*Ptot][gq pitch]                  */
    SZSNN_L_LQ_COUNTER,          /* uint32 [Ptot][D]                           */
    SZSNN_L_LQ_ENTRIES,          /* short2 [Ptot][D][ALIGN(MPS*D,32)]          */
    SZSNN_L_FIRED,               /* uint32 [Ptot][MPS]                         */
    SZSNN_L_FIRED_COUNT,         /* uint32 [Ptot]                              */
    SZSNN_L_FIRED_INPUT,         /* uint32 [Ptot][MPS/32]                      */
    SZSNN_L_FIRED_OUTPUT,        /* uint32 [Ptot][MPS/32]                      */
    SZSNN_L_INPUT_CURRENT,       /* float  [Ptot][MPS]                         */
    SZSNN_L_CURRENT,             /* float  [2][Ptot][MPS]                      */
    SZSNN_L_COUNT
};
typedef struct {
    uint32_t neuron_partitions, input_partitions, total_partitions;
    uint32_t group_pitch, group_step;
    uint64_t gq_pitch;            /* max incoming bundles of a partition */
    uint64_t bundles;             /* bundle rows incl. the unused row 0 */
    uint64_t bytes[SZSNN_L_COUNT];
} szsnn_layout_info;

int szsnn_layout_build(const szsnn_layout_consts* consts, const szsnn_layout_desc* desc,
                       szsnn_layout** out, char* err, size_t err_len);
int szsnn_layout_info_get(const szsnn_layout* L, szsnn_layout_info* info);
int szsnn_layout_array(const szsnn_layout* L, int which, void* dst, size_t dst_bytes);
int szsnn_layout_free(szsnn_layout* L);

/* ---------------------------------------------- 3. native network path --
 * Units: neurons 0..N-1, then sources N..N+P-1.  Synapses are rows per unit,
 * bucketed by delay m = 1..D (m = the reference's stored delay, user delay + 1):
 * bucket (s, m) = [row_ptr[s*D + m-1], row_ptr[s*D + m]).  A spike emitted at
 * step t over a delay-m synapse is integrated by the update of step t + m,
 * as in the reference (scatter_kernel.cl:154,207; gather_kernel.cl:55-58). */
enum {
    SZSNN_IF_CURR_EXP = 0,
    SZSNN_IF_COND_EXP = 1,
    SZSNN_IZHIKEVICH  = 2,
    SZSNN_POISSON     = 3,
    SZSNN_CONST_RATE  = 4
};
#define SZSNN_MAX_POPS 65536
#define SZSNN_POP_IZH_HALF_STEPS 1u

/* Parameter slots: IF_curr_exp 0 v_rest 1 cm 2 tau_m 3 tau_refrac 4 tau_syn_E
 * 5 tau_syn_I 6 i_offset 7 v_reset 8 v_thresh (IF_curr_exp_NeuronModel.hpp:12-23);
 * IF_cond_exp adds 9 e_rev_E 10 e_rev_I; Izhikevich 0 a 1 b 2 c 3 d;
 * Poisson 0 p (spike probability per step); Const_rate 0 rate (steps).
 * Times are in steps (dt folded, as the reference's kernels assume dt = 1).
 * State slots: IF*: 0 v 1 Ie|ge 2 Ii|gi 3 steps-since-spike; Izhikevich 0 v 1 u;
 * Const_rate 0 last. */
typedef struct {
    int32_t  model;
    uint32_t flags;
    int64_t  begin, end;
    float    p[12];
    const float* pn_host;   /* per-unit parameters SoA [slot][end-begin] (host), or NULL */
    uint64_t seed;          /* Poisson stream key */
} szsnn_pop_desc;

#define SZSNN_ACC_FLOAT 0u  /* fp32 atomic accumulation (order not fixed)          */
#define SZSNN_ACC_FIXED 1u  /* int64 fixed point, w*2^32 rounded: bit-reproducible */

typedef struct {
    int64_t  n_neurons, n_sources;
    int32_t  max_delay;             /* D, 1..1024 */
    int32_t  n_pops;                /* <= SZSNN_MAX_POPS */
    const szsnn_pop_desc* pops;     /* ranges disjoint, sorted by begin */
    uint64_t n_synapses;
    const uint64_t* row_ptr_host;   /* (N+P)*D+1, or NULL with szsnn_net_generate */
    const int32_t*  tgt_host;
    const float*    w_host;
    const float*    state_host[4];  /* initial state slots (length N+P) or NULL = 0 */
    uint32_t acc_mode;
    uint32_t graph_chunk;           /* steps per captured CUDA graph (0 = 100) */
    int64_t  raster_capacity;       /* reserved, 0 */
    const int32_t* group_host;      /* per-unit group id (e.g. the network of a batch), or NULL */
    int32_t  n_groups;              /* spike counters kept per group when group_host is set */
} szsnn_net_desc;

/* Fixed fan-out generator block (device-side; identical algorithm in the
 * test oracle): rows src_begin.. get `fanout` synapses with target
 * ~U{tgt range} (self excluded on request), w = w_sign*(w_lo + (w_hi-w_lo)*u),
 * delay ~U{d_lo..d_hi}, stored stably bucketed by delay. */
typedef struct {
    int64_t  src_begin, src_count;
    int64_t  tgt_begin, tgt_count;
    int32_t  fanout;
    int32_t  exclude_self;
    float    w_lo, w_hi, w_sign;
    int32_t  d_lo, d_hi;
    uint32_t stream;
    uint64_t syn_offset;
} szsnn_gen_block;

typedef struct {
    int64_t  steps_done;
    uint64_t events;          /* delivered synaptic events (non-zero weights) */
    uint64_t spikes;          /* spikes of neurons and sources */
    uint64_t graph_launches;
    uint64_t kernel_launches;
} szsnn_net_stats;

int szsnn_net_create(szsnn_ctx* ctx, const szsnn_net_desc* desc, szsnn_net** out);
int szsnn_net_generate(szsnn_net* net, const szsnn_gen_block* blocks, int n_blocks, uint64_t seed);
int szsnn_net_destroy(szsnn_net* net);
/* Simulation::stepAndFired(fInput) (Simulation.ipp:517-530): one step with
 * optional host forced-spike words and external current, fired words out. */
int szsnn_net_step(szsnn_net* net, const uint32_t* forced_host, const float* current_host,
                   uint32_t* fired_host);
/* No counterpart in the reference (one device per network, Context.cpp:211-213):
 * the exchange step of a network sharded by unit ranges across devices.
 * words_host ([words] spike words, host memory) holds the spikes that units
 * updated by other shards emitted in the step just done; they are appended
 * to this network's spike ring for that step and, in the overlapped order,
 * their delay-1 buckets delivered into the next step's inputs -- what the
 * update does for its own spikes.  Call it after each step, before the next. */
int szsnn_net_inject_spikes(szsnn_net* net, const uint32_t* words_host);
/* The units this network updates when it is one shard of a network split by
 * unit ranges: neurons [n_lo, n_hi) and sources [s_lo, s_hi); the others keep
 * their state and never spike here (their spikes arrive by
 * szsnn_net_inject_spikes).  Default: every unit. */
int szsnn_net_set_owned(szsnn_net* net, int64_t n_lo, int64_t n_hi, int64_t s_lo, int64_t s_hi);
/* `steps` steps in CUDA-graph chunks.  forced_host: [steps][words] or NULL;
 * raster_host: [steps][words] output spike words or NULL. */
int szsnn_net_run(szsnn_net* net, int64_t steps, const uint32_t* forced_host,
                  uint32_t* raster_host);
/* Same with device buffers: forced_dev [steps][words], current_dev [steps][N],
 * raster_dev [steps][words]; any may be NULL.  Asynchronous on the stream. */
int szsnn_net_run_device(szsnn_net* net, int64_t steps, const uint32_t* forced_dev,
                         const float* current_dev, uint32_t* raster_dev);
int szsnn_net_stats_get(szsnn_net* net, szsnn_net_stats* out);
/* spikes per group since creation (or the last reset): counts[n_groups] */
int szsnn_net_group_spikes(szsnn_net* net, uint64_t* counts, int reset);
/* state slot k (length N+P) copy out / in (checkpoint) */
int szsnn_net_get_state(szsnn_net* net, int slot, float* host);
int szsnn_net_set_state(szsnn_net* net, int slot, const float* host);
/* State monitor (no counterpart in the reference, whose print_vars.py reads the
 * whole state back every cycle): after every step of szsnn_net_step / run /
 * run_device, the state slots in slot_mask (bit k: slot k, 1..15) of the n_ids
 * units ids[] are appended on the device to a trace of `capacity` steps; steps
 * past the capacity are not recorded.  n_ids = 0 turns the monitor off.
 * Recording starts at the current step; one extra small kernel per step. */
int szsnn_net_set_monitor(szsnn_net* net, const int32_t* ids, int32_t n_ids, uint32_t slot_mask, int64_t capacity);
/* The trace since szsnn_net_set_monitor or the last read: out [steps][slots][n_ids]
 * fp32, slots in ascending order, at most max_steps; *steps_out = steps copied,
 * *dropped_out = steps run since the start that were not copied (past the
 * capacity or past max_steps).  Waits for the stream; recording then restarts
 * at the current step. */
int szsnn_net_monitor_read(szsnn_net* net, float* out, int64_t max_steps, int64_t* steps_out,
                           int64_t* dropped_out);
/* whole-simulation checkpoint: state, spike ring and clock into one blob */
int szsnn_net_checkpoint_size(szsnn_net* net, uint64_t* bytes);
int szsnn_net_checkpoint(szsnn_net* net, void* host_blob, uint64_t bytes);
int szsnn_net_restore(szsnn_net* net, const void* host_blob, uint64_t bytes);
/* copy the device CSR back (row_ptr (N+P)*D+1, tgt, w) -- checks the generator */
int szsnn_net_get_synapses(szsnn_net* net, uint64_t* row_ptr, int32_t* tgt, float* w);
/* scan the state slots for NaN/Inf: sets SZSNN_DEV_NONFINITE */
int szsnn_net_check_finite(szsnn_net* net, int* finite_out);
/* inputs integrated at the last step (debug/parity): in_exc, in_inh (N) */
int szsnn_net_last_inputs(szsnn_net* net, float* in_exc, float* in_inh);

/* per-kernel device time: `steps` replays of the current step's propagate and
 * update launches on scratch copies of the state (the network is unchanged),
 * timed with CUDA events on the stream; sums over the replays, in ms, and the
 * synaptic events one propagate launch delivers */
int szsnn_net_profile(szsnn_net* net, int64_t steps, double* propagate_ms, double* update_ms,
                      double* events_per_launch);
/* As szsnn_net_profile, plus the device time of `steps` replays of the whole
 * step (overlapped order: the fused k_step launch; classic: propagate +
 * update), the time every simulated step costs. */
int szsnn_net_profile_step(szsnn_net* net, int64_t steps, double* propagate_ms, double* update_ms, double* step_ms,
                           double* events_per_launch);
/* total_ms: device time (CUDA events on the stream) of the last szsnn_net_run /
 * szsnn_net_run_device; propagate/update: the last szsnn_net_profile */
int szsnn_net_timing(szsnn_net* net, double* propagate_ms, double* update_ms, double* total_ms);
/* launch shapes: propagate mode 0 = `group` lanes per (delay, spike) bucket
 * segment (4/8/16/32), mode 1 = warp-flattened walk over `group` items per
 * warp (8/16/32); propagate grid blocks (0 = 16 per SM); update block size
 * (threads, a multiple of 32 in 32..256; each thread updates 4 units) */
int szsnn_net_set_tuning(szsnn_net* net, int propagate_mode, int group, int propagate_blocks, int update_block);
/* Units each update thread handles per step (1..16; 0 = automatic: 4 while
 * the network gives at least four update blocks per SM, fewer below).  A
 * block's tile is update_block x units; fewer, longer blocks trade the
 * launch's trailing partial wave for longer blocks.  Results are identical
 * for every value. */
int szsnn_net_set_update_units(szsnn_net* net, int units_per_thread);
/* Update tiles: mode 0 = one tile per update block, a new block per tile each
 * step; mode 1 = persistent warp tiles: blocks_per_sm update blocks per SM
 * (0 = 2), each warp streaming 128-unit tiles through a two-stage ring of
 * bulk copies in shared memory and writing them back with bulk stores (for
 * networks of at most four populations; others keep mode 0); mode 2 =
 * persistent block tiles: the tiles of mode 0 taken in turn by as many update
 * blocks as stay resident (blocks_per_sm, or 0 = from the occupancy of the
 * launch).  Results are identical in every mode. */
int szsnn_net_set_update_tiles(szsnn_net* net, int mode, int blocks_per_sm);
/* Resident stepping (on = 1): szsnn_net_run / szsnn_net_run_device run each
 * chunk as one cooperative launch of `blocks` blocks (0 = one per SM) of
 * 1024 threads that keeps the neurons' state in shared memory across the
 * chunk's steps, with a bounded grid barrier between steps; in each block
 * `update_warps` warps (0 = 16) update its neuron and source words while the
 * other warps take their share of the far delivery.  Same step order,
 * arithmetic and results as the overlapped graphs (bit-identical in
 * fixed-point accumulation).  Needs the overlapped order, at most four
 * populations (IF_curr_exp, IF_cond_exp, Izhikevich neurons; Poisson
 * sources; shared or per-unit parameters), no state monitor, and a block's neuron state
 * within shared memory (about 1.6M IF neurons on one B200); otherwise
 * SZSNN_ERR_ARG with the reason, and a later run whose network no longer
 * qualifies fails with SZSNN_ERR_STATE.  szsnn_net_step and the profiling
 * calls keep the per-step launches.  A grid barrier that waits past its
 * bound records device error SZSNN_DEV_WAIT_TIMEOUT and ends the launch. */
int szsnn_net_set_resident(szsnn_net* net, int on, int update_warps, int blocks);
/* Step order.  1 (default): overlapped -- input buffers double-buffered by
 * step parity, delivery of delays >= 2 into step t+1 runs in the same launch
 * as update(t), and update(t) delivers the delay-1 bucket of its own
 * spikes.  0: classic -- propagate(t) delivers delays 1..D, then update(t)
 * (the reference's order, Simulation.ipp:471-496).  Results are identical in
 * fixed-point accumulation; switching mid-run rebuilds the next step's
 * inputs from the spike ring. */
int szsnn_net_set_overlap(szsnn_net* net, int overlap);

/* ------------------------------------------ differentiable IF_curr_exp ---
 * BPTT for a recurrent IF_curr_exp layer (no reference counterpart; the
 * forward rule is IF_curr_exp_update_kernel.cl:230-287 with dt folded to 1
 * and tau_refrac 0, the channel of a weight is its sign as in
 * gather_kernel.cl:172-178).  Inputs x_t are integrated in their step,
 * recurrent spikes one step later; y_t = alpha y_{t-1} + Wout^T s_t, outputs
 * ymax = max_t y_t (with its first argmax) and vsum = sum_t v_t.  The
 * backward is exact except dH/du, replaced by 1/(1 + beta|u - v_thresh|)^2
 * (beta <= 0: 0), with forward spikes kept.  The backward reads u from the
 * trajectory the forward stored in u_trace when the caller passes it again
 * (T*B*N floats: 1.28 GB at T 500, B 64, N 10,000), else recomputes u from
 * the checkpoints every `checkpoint_every` steps (the same kernel, so the
 * same u and gradients bit for bit).  All pointers are device pointers owned by
 * the caller (e.g. torch tensors); `workspace` holds
 * szsnn_bptt_workspace_bytes bytes.  Calls are asynchronous on `stream`. */
typedef struct {
    int32_t B, N, M, K, T, checkpoint_every;        /* trials (<= 64), neurons, inputs, readouts (<= 64), steps */
    float v_rest, cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I, i_offset, v_reset, v_thresh;  /* step units */
    float alpha;                                    /* readout leak factor */
    float beta;                                     /* surrogate slope */
    int64_t nnz;                                    /* recurrent synapses */
    const float* w_in;                              /* [M][N] */
    const int64_t* rec_row_ptr;                     /* [N+1] CSR of the recurrent weights, row = presynaptic */
    const int32_t* rec_col;                         /* [nnz] postsynaptic neuron */
    const float* rec_val;                           /* [nnz] */
    const float* w_out;                             /* [N][K] */
    const uint32_t* x_bits;                         /* [T][B][ceil(M/32)] input spike words */
    const float* v0;                                /* [B][N] initial membrane */
    uint32_t* spikes;                               /* [T][B][ceil(N/32)] out: spike words */
    float* ckpt;                                    /* [ceil(T/ck)][3][B][N] out: (Ie, Ii, v) checkpoints */
    float* ymax;                                    /* [B][K] out */
    int32_t* tmax;                                  /* [B][K] out */
    float* vsum;                                    /* [B][N] out */
    float* u_trace;                                 /* [T][B][N] forward out: pre-reset membrane, or NULL;
                                                       backward in: that trajectory (no recompute), or NULL */
    const float* g_ymax;                            /* [B][K] dL/dymax (backward), or NULL */
    const float* g_vsum;                            /* [B][N] dL/dvsum (backward), or NULL */
    float* dw_in;                                   /* [M][N] out (backward) */
    float* dw_rec;                                  /* [nnz] out (backward) */
    float* dw_out;                                  /* [N][K] out (backward) */
    double* phase_ms;                               /* host [4] or NULL: backward adds its device ms per phase
                                                       (recompute, recurrent term + dWrec, adjoint, dWin) */
    void* workspace;
    void* stream;                                   /* cudaStream_t */
} szsnn_bptt_desc;
int szsnn_bptt_workspace_bytes(const szsnn_bptt_desc* d, uint64_t* bytes);
int szsnn_bptt_forward(const szsnn_bptt_desc* d, char* err, size_t err_len);
int szsnn_bptt_backward(const szsnn_bptt_desc* d, char* err, size_t err_len);

/* ------------------------------------------------------ measured ceilings ---
 * No counterpart in the reference.  The step keeps its neuron state and input
 * accumulators in L2 across steps and does one fp32 reduction per synaptic
 * event at a random target, so its roofline denominators are on-chip rates,
 * measured here on the device of `ctx`: an L2-resident copy (two 16 MB
 * buffers, read + write bytes per second) and random `red.add.f32` into
 * 2 * n_targets floats (reductions per second).  Synchronous; allocates and
 * frees its own buffers. */
typedef struct {
    double  l2_copy_gbs;     /* read + write GB/s of the L2-resident copy        */
    int64_t l2_copy_bytes;   /* bytes of the two copy buffers                   */
    double  red_per_s;       /* random fp32 reductions per second               */
    int64_t red_targets;     /* floats the reductions land in                   */
} szsnn_peaks;
int szsnn_probe_peaks(szsnn_ctx* ctx, int64_t n_targets, szsnn_peaks* out);

/* ----------------------------------------- allocation-free single step ---
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- hosts that own and partition all of it (a fixed-budget pool or
 * arena, a framework's caching allocator) and forbid libraries from calling
 * cudaMalloc, or real-time loops that cannot take cudaMalloc's implicit device
 * synchronisation -- szsnn_step_static runs one propagate + update step of a
 * network held entirely in caller-provided device buffers (one neuron
 * population of a single model and parameter set, plus optional Poisson
 * sources).  The step's scratch (input accumulators and a small header) is a
 * file-scope static device array of fixed size inside the library, held by
 * every GPU that loads it until the process exits: at most
 * SZSNN_STATIC_MAX_NEURONS neurons, larger networks return SZSNN_ERR_LIMIT.
 * The first call on a device looks up the array's device address (make it
 * before any stream capture).  Every call shares the array and clears what
 * must start at zero; calls that overlap on the GPU race on it and must be
 * serialised by the caller.  The call is asynchronous on `stream`; the
 * population table and the step number travel as kernel parameters, so
 * nothing is read from this struct after the call returns.  Device-side
 * errors (a synapse target outside the neurons, a full ring slot) are
 * recorded in `error_word`, which is required: zero it before the first
 * call; the first error stays there until the caller clears it. */
#define SZSNN_STATIC_MAX_NEURONS 262144
typedef struct {
    int64_t  n_neurons, n_sources;
    int32_t  max_delay;
    int64_t  step;              /* absolute step number of this call */
    int32_t  model;             /* SZSNN_IF_CURR_EXP, SZSNN_IF_COND_EXP or SZSNN_IZHIKEVICH */
    uint32_t flags;             /* SZSNN_POP_IZH_HALF_STEPS */
    float    params[12];        /* one parameter set, slots as szsnn_pop_desc */
    float    source_p;          /* spike probability per step of every Poisson source */
    uint64_t seed;
    const uint64_t* row_ptr;    /* device, (N+P)*D+1, delay-bucketed rows */
    const int32_t*  syn;        /* device, (target, fp32 weight bits) pairs */
    float*    state[4];         /* device, N+P each, slots as szsnn_pop_desc */
    uint32_t* ring_cnt;         /* device, D+1, zero before the first step */
    int32_t*  ring_ids;         /* device, (D+1)*(N+P) */
    uint32_t* fired_words;      /* device out, (N+P+31)/32 spike words, or NULL */
    uint32_t* error_word;       /* device in/out, 2 words (code, info); required, sticky */
    void*     stream;           /* cudaStream_t, NULL = legacy default stream */
} szsnn_static_step;
int szsnn_step_static(const szsnn_static_step* s, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif
