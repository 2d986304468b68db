/*
 * oracle.h -- CPU restatement ("Oracle A") of SZSNN's clock-driven simulation step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (szsnn_b200/, include/)
 * links or calls this library; only tests/, the smoke check and the bench's
 * cpu_baseline / reference arm use it, as the checker.  It is plain C, compiled
 * with -ffp-contract=off and FTZ/DAZ on (the reference builds its kernels with
 * -cl-denorms-are-zero and -cl-single-precision-constant,
 * szsnn1.1/src/Simulation.ipp:13-15, models/neuron_model_traits.hpp:42-43).
 *
 * What it restates (all file:line are relative to the reference project):
 *   IF_curr_exp update   szsnn1.1/src/cl/IF_curr_exp_update_kernel.cl:224-298
 *   Izhikevich update    szsnn1.1/src/cl/Izhikevich_update_kernel.cl:214-290
 *   Const_rate update    szsnn1.1/src/cl/Const_rate_update_kernel.cl:205-230
 *   gather (exc/inh split by weight sign, w == 0 skipped)
 *                        szsnn1.1/src/cl/gather_kernel.cl:150-183
 *   scatter delay rule   szsnn1.1/src/cl/scatter_kernel.cl:137-171,204-213,325-345
 *                        + gather read slot gather_kernel.cl:55-58,104:
 *                        a spike emitted by update(c) over a synapse whose stored
 *                        delay is m (= user delay + 1, NetworkGraph.ipp:431)
 *                        is integrated by update(c + m).
 *   step order           szsnn1.1/src/Simulation.ipp:471-496 (gather, update +
 *                        input, scatter)
 * Extensions with no reference counterpart (their parity is pinned only to the
 * equations stated here): IF_cond_exp, Poisson sources, Izhikevich 2 x 0.5
 * half-steps, fixed-point accumulation, arbitrary delay depth, fp64 twin.
 *
 * Network form: rows = sources (neurons 0..N-1 then sources N..N+P-1), each row
 * bucketed by delay m = 1..D: bucket (s, m) spans
 * [row_ptr[s*D + m-1], row_ptr[s*D + m]) of (tgt[], w[]).
 */
#ifndef SZSNN_ORACLE_H
#define SZSNN_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_POPS 16

enum {
    ORC_IF_CURR_EXP = 0,
    ORC_IF_COND_EXP = 1,
    ORC_IZHIKEVICH  = 2,
    ORC_POISSON     = 3,
    ORC_CONST_RATE  = 4
};

/* flags */
#define ORC_IZH_HALF_STEPS 1u

/* Parameter slots (per model), same numbering as the product:
 * IF_curr_exp : 0 v_rest 1 cm 2 tau_m 3 tau_refrac 4 tau_syn_E 5 tau_syn_I
 *               6 i_offset 7 v_reset 8 v_thresh   (IF_curr_exp_NeuronModel.hpp:12-23)
 * IF_cond_exp : the nine above + 9 e_rev_E 10 e_rev_I
 * Izhikevich  : 0 a 1 b 2 c 3 d                    (Izhikevich_NeuronModel.hpp:82-88)
 * Poisson     : 0 p (spike probability per step)
 * Const_rate  : 0 rate (steps)                     (Const_rate_InputModel.hpp:140-143)
 * State slots : IF*: 0 v 1 Ie|ge 2 Ii|gi 3 fired (steps since spike, float)
 *               Izhikevich: 0 v 1 u ; Const_rate: 0 last */
typedef struct {
    int32_t  model;
    uint32_t flags;
    int64_t  begin, end;      /* unit id range */
    float    p[12];           /* uniform parameters */
    const float* pn;          /* per-unit parameters SoA [slot][end-begin], or NULL */
    uint64_t seed;            /* Poisson */
} orc_pop;

typedef struct {
    int64_t  n_neurons, n_sources;
    int32_t  max_delay;
    int32_t  n_pops;
    orc_pop  pops[ORC_MAX_POPS];
    const uint64_t* row_ptr;  /* (N+P)*D + 1 */
    const int32_t*  tgt;
    const float*    w;
} orc_net;

/* accumulate modes */
#define ORC_ACC_FLOAT 0   /* fp sums in canonical order: m = 1..D, source ascending, bucket order */
#define ORC_ACC_FIXED 1   /* int64 sums of llrintf(w * 2^32), converted back once per step */

/*
 * Run `steps` steps starting at absolute step t0.
 *  state[k]    : per-unit state slot k, length N+P (fp32 run) -- updated in place
 *  hist        : spike history ring, D slots x words(N+P) uint32, in/out
 *  ext_current : [steps][N] external current (isInputCurrent), or NULL
 *  forced      : [steps][words(N+P)] forced-spike bits (isInputFiring), or NULL
 *  raster      : [steps][words(N+P)] output spike bits, or NULL
 *  in_exc/in_inh (optional, length N): the inputs integrated at the last step
 * Returns delivered synaptic events (non-zero weights).
 */
uint64_t orc_run_f32(const orc_net* net, float* state[4], uint32_t* hist,
                     int64_t t0, int64_t steps,
                     const float* ext_current, const uint32_t* forced,
                     uint32_t* raster, int acc_mode, int nthreads,
                     float* in_exc_out, float* in_inh_out);

/* fp64 twin: state in double; weights/params widened from fp32 */
uint64_t orc_run_f64(const orc_net* net, double* state[4], uint32_t* hist,
                     int64_t t0, int64_t steps,
                     const float* ext_current, const uint32_t* forced,
                     uint32_t* raster, int nthreads);

/* fixed fan-out network generator (identical algorithm on device) */
typedef struct {
    int64_t  src_begin, src_count;   /* rows generated */
    int64_t  tgt_begin, tgt_count;   /* uniform target range */
    int32_t  fanout;
    int32_t  exclude_self;           /* skip tgt == src (when ranges overlap) */
    float    w_lo, w_hi, w_sign;     /* w = w_sign * (w_lo + (w_hi - w_lo) * u24) */
    int32_t  d_lo, d_hi;             /* delay m ~ U{d_lo..d_hi} */
    uint32_t stream;                 /* block stream id */
    uint64_t syn_offset;             /* first synapse slot of row src_begin */
} orc_gen_block;

/* Fill tgt/w for the block and the row_ptr entries of its rows (row_ptr is
 * sized (N+P)*D+1; the caller sets row_ptr[(N+P)*D]). */
void orc_gen_fixed_fanout(const orc_gen_block* b, uint64_t seed, int32_t max_delay,
                          uint64_t* row_ptr, int32_t* tgt, float* w);

/* Philox4x32-10 block, exposed for the RNG parity test */
void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
