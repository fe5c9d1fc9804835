/*
 * ctl_oracle.h -- CPU oracle for the cuTauLeaping simulation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the cutauleaping_b200
 * package, its CUDA library or its CLI) includes, links or calls this code.
 * It is used by tests/, by __graft_entry__.smoke() as the checker, and by
 * bench.py as the timed CPU baseline ("port" of the reference routine).
 *
 * What it restates (reference file:line, paths inside aresio/cuTauLeaping):
 *   PreCalculations          2phase_n-tau-leaping.cu:1568-2093  (one Cao leap or SSA hand-off)
 *   CalculatePropensity      2phase_n-tau-leaping.cu:1443-1470  (DEV_FLATTEN_MATRIX_CONST)
 *   test_update              2phase_n-tau-leaping.cu:1300-1351  (negative-population test)
 *   check_time_instant       2phase_n-tau-leaping.cu:1507-1562  (interpolated samples)
 *   EventualSSASteps         2phase_n-tau-leaping.cu:2099-2273  (bursts of 100 SSA steps)
 *   LightweightSSA           2phase_n-tau-leaping.cu:2280-2454  (forced-SSA mode)
 *   HOR / HORtype            2phase_n-tau-leaping.cu:402-432
 *   stoichiometry flattening 2phase_n-tau-leaping.cu:122-400
 *
 * The reference draws its random numbers from cuRAND's XORWOW device API,
 * which is not part of the reference sources, and seeds it from time(NULL)
 * (kernel.cu:176).  Its trajectories are therefore not reproducible, and
 * parity with it is statistical.  This oracle instead fixes one canonical
 * arithmetic contract that the CUDA kernels must reproduce bit for bit:
 *   - Philox4x32-10 (Salmon et al., SC'11) keyed by (seed) with counter
 *     (block, tag, step, sim);
 *   - own log/exp (Cody-Waite reduction + atanh / Taylor series), own
 *     Poisson sampler (sequential inversion for lambda < 10, Hormann 1993
 *     PTRS otherwise);
 *   - FP32 propensities, FP64 sums arranged as a fixed binary tree over the
 *     reactions (padded to a power of two), FP64 simulated time.
 * The oracle is pinned separately against the reference binary's own output
 * (statistical fixtures in tests/golden) and against an exact FP64 Gillespie
 * direct method (ctlo_gillespie below).
 */
#ifndef CTL_ORACLE_H
#define CTL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Switches that turn OFF one reference quirk each (0 = reference behaviour). */
enum {
    CTLO_FORCE_SSA = 1u << 0,  /* kernel.cu:115, LightweightSSA only              */
    CTLO_Q1_OFF    = 1u << 1,  /* signed interpolation (ref clamps negative deltas, tau.cu:1538-1541) */
    CTLO_Q2_OFF    = 1u << 2,  /* mask PROP[0] in the critical pick (ref tau.cu:1997) */
    CTLO_Q3_OFF    = 1u << 3,  /* keep the critical firing on a rejection retry (ref drops it, tau.cu:2044-2046) */
    CTLO_Q4_OFF    = 1u << 4,  /* reject only on final negatives (ref: any intermediate, tau.cu:1327-1329) */
    CTLO_Q5_OFF    = 1u << 5,  /* tau1 over feed-masked F instead of full V (ref tau.cu:1860-1922) */
    CTLO_Q6_OFF    = 1u << 6,  /* critical iff floor(X/L) < nc (ref: 0 < floor < nc, tau.cu:1731) */
    CTLO_Q9_OFF    = 1u << 7,  /* use the sigma bound even when mu == 0 (ref skips, tau.cu:1904-1911) */
    CTLO_Q10_OFF   = 1u << 8   /* A0==0: fill with the current state (ref copies the last sample, tau.cu:1665-1697) */
};

/* Per-simulation status codes (same values as the product's ctl_sim_status). */
enum { CTLO_SIM_OK = 0, CTLO_SIM_STEP_LIMIT = 1, CTLO_SIM_OVERFLOW = 2, CTLO_SIM_ATTEMPT_LIMIT = 3 };

typedef struct {
    double   t_final;     /* simulated time when the simulation stopped          */
    uint64_t firings;     /* sum of K over accepted leaps + executed SSA steps   */
    uint32_t status;      /* CTLO_SIM_*                                          */
    uint32_t steps;       /* step counter (decisions + SSA steps)                */
    uint32_t leaps;       /* accepted tau-leaps                                  */
    uint32_t ssa_steps;   /* executed SSA steps                                  */
    uint32_t rejections;  /* negative-population rejections (tau halvings)       */
    uint32_t pad;
} ctlo_info;

typedef struct ctlo_model ctlo_model;

/* left/right: dense [R][S] stoichiometry; feed: [S] (nonzero = species held
 * constant, the M_feed file).  tvec: sample instants (ns); cs: sampled species.
 * Returns NULL on invalid input. */
ctlo_model* ctlo_model_new(int S, int R, const int32_t* left, const int32_t* right,
                           const int32_t* feed, int ns, const double* tvec,
                           int s_out, const int32_t* cs,
                           float eps, uint32_t nc, double ssa_factor, uint32_t ssa_steps,
                           uint32_t flags, uint64_t seed, uint32_t max_steps);
void ctlo_model_free(ctlo_model* m);
void ctlo_model_hor(const ctlo_model* m, uint8_t* hor, uint8_t* hort);

/* One simulation: X0[S], c[R] (FP32 rate constants), out[ns][s_out]. */
int ctlo_simulate(const ctlo_model* m, uint32_t sim, const int32_t* X0, const float* c,
                  uint32_t* out, ctlo_info* info);
/* Exact FP64 Gillespie direct method (independent oracle). */
int ctlo_gillespie(const ctlo_model* m, uint32_t sim, const int32_t* X0, const float* c,
                   uint32_t* out, ctlo_info* info);
/* n simulations on nthreads host threads; mode 0 = canonical tau-leaping,
 * 1 = Gillespie.  X0 [n][S], c [n][R], out [n][ns][s_out], info [n]. */
int ctlo_run_batch(const ctlo_model* m, int n, uint32_t sim_base, const int32_t* X0,
                   const float* c, uint32_t* out, ctlo_info* info, int nthreads, int mode);

/* Primitives exposed for known-answer and distribution tests. */
void     ctlo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double   ctlo_log(double x);
float    ctlo_logf(float x);
double   ctlo_exp(double x);
double   ctlo_logfact(double k);
uint32_t ctlo_poisson(double lam, uint64_t seed, uint32_t sim, uint32_t step,
                      uint32_t attempt, uint32_t r);

#ifdef __cplusplus
}
#endif
#endif
