/*
 * oracle.c -- CPU restatement of the SZSNN simulation step (see oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, smoke() and bench.py's cpu_baseline
 * and reference arm as the checker; never linked into the product.
 *
 * Build (oracle/build.py): gcc -O2 -fopenmp -ffp-contract=off -fno-fast-math
 * -shared -fPIC.  FTZ/DAZ is switched on at entry of each run, mirroring the
 * reference's -cl-denorms-are-zero (szsnn1.1/src/Simulation.ipp:14).
 */
#include "oracle.h"
#include "philox.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>
#include <pmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* FTZ/DAZ for the duration of one call; the caller's MXCSR is restored */
static unsigned orc_ftz_on(void)
{
    unsigned saved = _mm_getcsr();
    _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
    _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
    return saved;
}

void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    orc_u32x4 r = orc_philox(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
    memcpy(out, r.v, sizeof(r.v));
}

static inline int64_t orc_words(int64_t n) { return (n + 31) / 32; }

static inline const orc_pop* orc_find_pop(const orc_net* net, int64_t id)
{
    for (int i = 0; i < net->n_pops; ++i)
        if (id >= net->pops[i].begin && id < net->pops[i].end) return &net->pops[i];
    return NULL;
}

static inline float orc_param(const orc_pop* p, int slot, int64_t id)
{
    if (p->pn) return p->pn[(int64_t)slot * (p->end - p->begin) + (id - p->begin)];
    return p->p[slot];
}

/* Poisson draw: spike iff u24(philox) < p, counter = index within the
 * population (no reference counterpart) */
static inline int orc_poisson_fires(uint64_t seed, int64_t idx, int64_t step, float p)
{
    orc_u32x4 r = orc_philox((uint32_t)idx, (uint32_t)step, (uint32_t)((uint64_t)step >> 32),
                             ORC_STREAM_POISSON, (uint32_t)seed, (uint32_t)(seed >> 32));
    return orc_u24(r.v[0]) < p;
}

/* ---- fixed fan-out generator ------------------------------------------- */
/* Rows are independent (row r owns synapses base + [0, F)), so they are
 * generated in parallel; each thread keeps its own delay histogram. */
void orc_gen_fixed_fanout(const orc_gen_block* b, uint64_t seed, int32_t D,
                          uint64_t* row_ptr, int32_t* tgt, float* w)
{
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const int F = b->fanout;
#pragma omp parallel
    {
    uint32_t* cnt = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(D + 1));
#pragma omp for schedule(static, 1024)
    for (int64_t r = 0; r < b->src_count; ++r) {
        const int64_t s = b->src_begin + r;
        const uint64_t base = b->syn_offset + (uint64_t)r * (uint64_t)F;
        memset(cnt, 0, sizeof(uint32_t) * (size_t)(D + 1));
        /* pass 1: delay histogram */
        for (int k = 0; k < F; ++k) {
            orc_u32x4 x = orc_philox((uint32_t)r, (uint32_t)k, b->stream, ORC_STREAM_GEN, k0, k1);
            int m = b->d_lo + (int)orc_bounded(x.v[2], (uint32_t)(b->d_hi - b->d_lo + 1));
            cnt[m] += 1;
        }
        /* bucket starts */
        uint64_t acc = base;
        for (int m = 1; m <= D; ++m) {
            row_ptr[s * D + (m - 1)] = acc;
            acc += cnt[m];
            cnt[m] = 0;
        }
        /* pass 2: stable placement by delay */
        for (int k = 0; k < F; ++k) {
            orc_u32x4 x = orc_philox((uint32_t)r, (uint32_t)k, b->stream, ORC_STREAM_GEN, k0, k1);
            int64_t t;
            if (b->exclude_self && s >= b->tgt_begin && s < b->tgt_begin + b->tgt_count) {
                t = b->tgt_begin + orc_bounded(x.v[0], (uint32_t)(b->tgt_count - 1));
                if (t >= s) t += 1;
            } else {
                t = b->tgt_begin + orc_bounded(x.v[0], (uint32_t)b->tgt_count);
            }
            float span = b->w_hi - b->w_lo;
            float mag = b->w_lo + span * orc_u24(x.v[1]);
            float wv = b->w_sign * mag;
            int m = b->d_lo + (int)orc_bounded(x.v[2], (uint32_t)(b->d_hi - b->d_lo + 1));
            uint64_t pos = row_ptr[s * D + (m - 1)] + cnt[m]++;
            tgt[pos] = (int32_t)t;
            w[pos] = wv;
        }
    }
    free(cnt);
    }
}

/* ---- the step, instantiated for fp32 and fp64 --------------------------- */
#define REAL float
#define SUFFIX f32
#include "oracle_step.inc"
#undef REAL
#undef SUFFIX

#define REAL double
#define SUFFIX f64
#define ORC_F64 1
#include "oracle_step.inc"
#undef ORC_F64
#undef REAL
#undef SUFFIX
