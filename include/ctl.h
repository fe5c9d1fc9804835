/*
 * ctl.h -- C ABI of cutauleaping_b200, a B200-native (sm_100a) drop-in for
 * the simulation path of aresio/cuTauLeaping.
 *
 * The reference has no library API: its boundary is the process command
 * line (kernel.cu:74-119), the input-folder text format
 * (2phase_n-tau-leaping.cu:57-1261) and one output file per simulation
 * (2phase_n-tau-leaping.cu:3431-3507).  This header is the C ABI beneath
 * that boundary; the `cutauleaping` CLI is a thin wrapper over it, and any
 * host language binds it through its C FFI.
 *
 * Conventions
 *   - Every entry point returns ctl_status; none calls exit().
 *   - Host buffers belong to the caller.  Device tables live inside the
 *     opaque ctl_model and are freed by ctl_model_free().
 *   - Per-simulation arrays are simulation-major: X0 [n][S], c [n][R],
 *     samples [n][ns][s_out] (uint32), info [n].
 *   - Results depend only on (model, rows, seed, sim_base, flags); launch
 *     shape, grouping and autotuning never change a single bit.
 *   - One run at a time per (model, device): runs share the model's queue
 *     counter on that device.
 */
#ifndef CTL_H
#define CTL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CTL_OK = 0,
    CTL_ERR_IO = 1,          /* a file could not be opened / read / written        */
    CTL_ERR_PARSE = 2,       /* malformed number or line in an input file          */
    CTL_ERR_SHAPE = 3,       /* inconsistent sizes (rows, columns, species ids)    */
    CTL_ERR_CUDA = 4,        /* CUDA runtime error (message in ctl_last_error())   */
    CTL_ERR_OOM = 5,         /* host or device allocation failed                    */
    CTL_ERR_STEP_LIMIT = 6,  /* at least one simulation ended with a non-OK status */
    CTL_ERR_TIMEOUT = 7,     /* reserved: bounded device waits gave up             */
    CTL_ERR_ARG = 8          /* invalid argument                                   */
} ctl_status;

/* Which input check failed, beside the status of the last failure
 * (ctl_last_error_detail): the cases for which the reference's reader exits
 * with its own code (2phase_n-tau-leaping.cu:598, 630, 646, 1139). */
typedef enum {
    CTL_DETAIL_NONE = 0,
    CTL_DETAIL_MX0_UNREADABLE = 1, /* MX_0 missing or unreadable (reference: exit -6)        */
    CTL_DETAIL_ROWS_SHORT = 2,     /* fewer MX_0 rows than offset + threads*blocks (-4)      */
    CTL_DETAIL_MX0_ROW = 3,        /* an MX_0 row of the wrong length or a bad entry (-5)    */
    CTL_DETAIL_TARGET_ASSIGN = 4   /* tts_vector does not cover threads*blocks (-10)         */
} ctl_error_detail;

/* Per-simulation status (ctl_sim_info.status). */
typedef enum {
    CTL_SIM_OK = 0,
    CTL_SIM_STEP_LIMIT = 1,     /* step counter reached ctl_run_cfg.max_steps        */
    CTL_SIM_OVERFLOW = 2,       /* a population exceeded INT32_MAX                   */
    CTL_SIM_ATTEMPT_LIMIT = 3   /* 1024 consecutive negative-population rejections   */
} ctl_sim_status;

/* Switches that turn OFF one reference quirk each; 0 reproduces the
 * reference algorithm (2phase_n-tau-leaping.cu line numbers in brackets). */
enum {
    CTL_FORCE_SSA = 1u << 0, /* exact SSA only, LightweightSSA [2280-2454]       */
    CTL_Q1_OFF = 1u << 1,    /* signed interpolation of samples [1538-1541]      */
    CTL_Q2_OFF = 1u << 2,    /* mask PROP[0] in the critical pick [1997]         */
    CTL_Q3_OFF = 1u << 3,    /* keep the critical firing on retry [2044-2046]    */
    CTL_Q4_OFF = 1u << 4,    /* reject on final negatives only [1327-1329]       */
    CTL_Q5_OFF = 1u << 5,    /* tau1 over feed-masked F, not V [1860-1922]       */
    CTL_Q6_OFF = 1u << 6,    /* critical iff floor(X/L) < nc [1731]              */
    CTL_Q9_OFF = 1u << 7,    /* sigma bound also when mu == 0 [1904-1911]        */
    CTL_Q10_OFF = 1u << 8    /* A0 == 0 fills with the current state [1665-1697] */
};

typedef struct ctl_model ctl_model;
typedef struct ctl_target ctl_target;
typedef struct ctl_graph ctl_graph;

typedef struct {
    int32_t S, R, P;            /* species, reactions, tree width (pow2 >= R)   */
    int32_t ns, s_out;          /* sample instants, sampled species             */
    int32_t nnz_left, nnz_var, nnz_feared, nnz_dep;
    double tmax;                /* last sample instant = simulated end time     */
} ctl_model_dims;

typedef struct {
    uint64_t seed;        /* Philox key; the reference used time(NULL) (kernel.cu:176) */
    float eps;            /* Cao epsilon, 0.03 (2phase_n-tau-leaping.cuh:76)           */
    uint32_t nc;          /* critical threshold, 10 (2phase_n-tau-leaping.cuh:75)      */
    double ssa_factor;    /* SSA hand-off when tau1 < ssa_factor/A0, 10 (tau.cu:1935)  */
    uint32_t ssa_steps;   /* SSA burst length, 100 (kernel.cu:83)                      */
    uint32_t flags;       /* CTL_FORCE_SSA | CTL_Q*_OFF                                */
    uint32_t max_steps;   /* per-simulation step cap (CTL_SIM_STEP_LIMIT)              */
    uint32_t sim_base;    /* global index of row 0 (the reference's `offset`)          */
    int32_t device;       /* CUDA device ordinal                                       */
    int32_t group;        /* lanes per simulation: 1..256, a power of two (above 32: whole
                             warps per simulation); 0 = library choice                */
    int32_t threads;      /* threads per block; 0 = autotune                           */
    int32_t uniform_rates;/* 1: every row of c equals row 0 (one shared copy per block);
                             ctl_run detects this itself, device calls take it as given */
    int32_t ssa_budget;   /* SSA steps per simulation and scheduling round (0 = 16; 8
                             when the batch fits in one wave of resident simulations) */
    int32_t dec_budget;   /* leap decisions per simulation and round (0 = 1; 2 for
                             groups of more than 32 lanes)                            */
    int32_t min_blocks;   /* register budget: kernel variant compiled for this many resident
                             256-thread blocks per SM (2: up to 128 registers per thread,
                             3: 80, 4: 64); 0 = library choice (autotuned, else 3 for
                             groups of 8+ lanes whose slots fit three blocks, else 2;
                             1 for the register-resident sweep, whose kernel compiled for
                             the network takes the budget given here; 1 is valid for that
                             sweep only) */
    int32_t sched;        /* scheduling: 1 = block rounds regrouping simulations by phase
                             (the register-resident sweep moves their state through shared
                             memory), 2 = warp-local (no block barriers; warp lockstep);
                             0 = library choice                                       */
    int32_t warp_sims;    /* register-resident sweep for tiny networks (at most 16 reactions,
                             8 species and sampled species, 3 reactant entries per reaction),
                             one thread per simulation: simulations per warp, 1..32 (with
                             sched 1, block rounds that regroup the simulations by phase,
                             the live simulations per warp of a block on average); 0 =
                             library choice (used for such networks unless `group` is
                             set); -1 = never (shared-memory sweep)                    */
    int32_t spec;         /* kernels compiled at run time for this network (NVRTC, sm_100a;
                             the library's own kernels when NVRTC is absent; same bits
                             either way): 0 = library choice (register-resident sweep:
                             always; shared-memory sweep: batches of at least 4,096
                             simulations, where the seconds of compilation, once per
                             process and network geometry, pay off), 1 = whenever
                             possible, -1 = never                                    */
} ctl_run_cfg;

typedef struct {
    double t_final;
    uint64_t firings;     /* sum of K over accepted leaps + executed SSA steps */
    uint32_t status;      /* ctl_sim_status                                    */
    uint32_t steps, leaps, ssa_steps, rejections, pad;
} ctl_sim_info;

typedef struct {
    int32_t group, threads, blocks, slots_per_block;
    int32_t smem_bytes, regs_per_thread, blocks_per_sm, sm_count;
    int32_t min_blocks;   /* register budget of the kernel variant (ctl_run_cfg.min_blocks) */
    int32_t sched;        /* scheduling mode (ctl_run_cfg.sched) */
    int32_t ssa_budget, dec_budget;  /* work per simulation and round */
    int32_t warp_sims;    /* simulations per warp of the register-resident sweep, 0 when the
                             shared-memory sweep runs (ctl_run_cfg.warp_sims) */
    int32_t specialized;  /* 1 when the sweep runs a kernel compiled for this network  */
} ctl_launch_info;

/* ---- errors ------------------------------------------------------------ */
const char* ctl_status_str(ctl_status s);
/* Message of the last failure on the calling thread ("" if none). */
const char* ctl_last_error(void);
/* ctl_error_detail of the last failure on the calling thread
 * (CTL_DETAIL_NONE when the failure has no finer code). */
int32_t ctl_last_error_detail(void);

/* ---- models -------------------------------------------------------------- */
/* Replaces first_pass + read_stoichiometry + read_instants
 * (tau.cu:90-120, 122-457, 932-1053): reads left_side, right_side, M_feed
 * (optional), t_vector and cs_vector (optional) from `folder`. */
ctl_status ctl_model_load(const char* folder, ctl_model** out);
/* Same model from dense arrays: left/right [R][S], feed [S] or NULL,
 * tvec [ns], cs [s_out] or NULL (all species). */
ctl_status ctl_model_create(int32_t S, int32_t R, const int32_t* left, const int32_t* right,
                            const int32_t* feed, int32_t ns, const double* tvec,
                            int32_t s_out, const int32_t* cs, ctl_model** out);
void ctl_model_free(ctl_model* m);
ctl_status ctl_model_dims_get(const ctl_model* m, ctl_model_dims* dims);
/* HOR / HORtype per species (tau.cu:402-432). */
ctl_status ctl_model_hor(const ctl_model* m, uint8_t* hor, uint8_t* hort);

/* Replaces read_quantities_offset + read_parameters_offset (tau.cu:570-649,
 * 717-782): rows [offset, offset+n) of MX_0 and c_matrix.  X0 [n][S] and
 * c [n][R] are caller buffers (rate constants stored FP32). */
ctl_status ctl_rows_load(const char* folder, int32_t S, int32_t R, uint32_t offset,
                         uint32_t n, int32_t* X0, float* c);

/* ---- simulation ---------------------------------------------------------- */
void ctl_run_cfg_default(ctl_run_cfg* cfg);
/* Replaces the host loop kernel.cu:155-345 (setup_random, PrepareVariables,
 * PreCalculations / EventualSSASteps / LightweightSSA, ParallelVoting) with
 * one persistent sweep.  Host buffers in and out; copies are inside the call.
 * Returns CTL_ERR_STEP_LIMIT if any simulation ended with a non-OK status. */
ctl_status ctl_run(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* X0,
                   const float* c, uint32_t* samples, ctl_sim_info* info);
/* The same sweep on device buffers, enqueued on `stream` (cudaStream_t). */
ctl_status ctl_run_device(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                          const int32_t* d_X0, const float* d_c, uint32_t* d_samples,
                          ctl_sim_info* d_info, void* stream);
/* Launch shape the sweep would use (after autotuning when cfg asks for it). */
ctl_status ctl_launch_query(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                            ctl_launch_info* li);

/* Diagnostics (no counterpart in the reference; no device work): the CUDA
 * source the library hands to NVRTC to compile the shared-memory sweep for
 * this network with `group` lanes per simulation (capped at the tree's
 * leaves) in register budget `min_blocks` (2, 3 or 4) -- see
 * ctl_run_cfg.spec.  *len receives the source's length; with buf != NULL
 * and cap > *len the source is copied there, NUL-terminated, else
 * CTL_ERR_SHAPE (call again with a larger buffer). */
ctl_status ctl_spec_source(const ctl_model* m, int32_t group, int32_t min_blocks, char* buf, size_t cap,
                           size_t* len);

/* The same sweep as ctl_run_device, for callers that cannot allocate device
 * memory (an application whose device memory comes only from its own pool,
 * a host that has fixed its device-memory budget, a layer that must not grow
 * memory behind its caller).  No counterpart in the reference.  The model
 * tables and the work-queue ticket live in a fixed 1 MiB array inside the
 * library instead of a cudaMalloc'd copy; models whose tables need more are
 * rejected with CTL_ERR_SHAPE.  The call allocates nothing: no cudaMalloc,
 * no cudaFree, no allocating library routine.  The first call on a device
 * looks up the array's device address (make it before any stream capture).
 * Every call reuses the same array and leaves its contents behind, so calls
 * whose work overlaps on the GPU (other streams, other threads) race: issue
 * them one after another. */
ctl_status ctl_run_device_noalloc(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                                  const int32_t* d_X0, const float* d_c, uint32_t* d_samples,
                                  ctl_sim_info* d_info, void* stream);

/* Measured autotuner: times the library's own plan and candidate shapes
 * (lanes per simulation, threads per block, scheduling, register budget,
 * per-round budgets) on the first `sample` simulations of the batch on
 * device buffers -- at least four waves of resident simulations, or the
 * whole batch -- and caches the fastest; later calls with
 * group == threads == 0 use it.  Never changes results. */
ctl_status ctl_autotune(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* d_X0,
                        const float* d_c, uint32_t sample, ctl_launch_info* best);

/* One CUDA graph holding the whole sweep (queue reset + persistent kernel);
 * replay with ctl_graph_launch.  Buffers are bound at creation. */
ctl_status ctl_graph_create(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n,
                            const int32_t* d_X0, const float* d_c, uint32_t* d_samples,
                            ctl_sim_info* d_info, void* stream, ctl_graph** out);
/* An uneven batch as one sweep: `count` batches (each its own model, run
 * configuration, rows and output buffers on device) captured as parallel
 * branches of ONE CUDA graph, so that the kernels share the GPU and one
 * batch's latency-bound tail overlaps the others' work.  Replaces running the
 * reference once per batch (its host loop, kernel.cu:242-345).  Every cfg
 * names the same device; a model appears at most once (its work-queue
 * ticket is per model and device). */
ctl_status ctl_graph_create_multi(uint32_t count, ctl_model* const* models, const ctl_run_cfg* cfgs,
                                  const uint32_t* n, const int32_t* const* d_X0, const float* const* d_c,
                                  uint32_t* const* d_samples, ctl_sim_info* const* d_info, void* stream,
                                  ctl_graph** out);
ctl_status ctl_graph_launch(ctl_graph* g, void* stream);
void ctl_graph_free(ctl_graph* g);

/* ---- output -------------------------------------------------------------- */
/* WriteDynamics2 (tau.cu:3431-3469): file <path_prefix>_<first_id + i> per
 * simulation, rows "t<TAB>x..." with iostream default formatting. */
ctl_status ctl_write_dynamics(const ctl_model* m, const char* path_prefix, uint32_t n,
                              const uint32_t* samples, uint32_t first_id, int32_t nthreads);
/* PrintDynamics2 (tau.cu:3472-3507): the same rows to stdout, a blank line
 * after each simulation. */
ctl_status ctl_print_dynamics(const ctl_model* m, uint32_t n, const uint32_t* samples);
/* One binary file for the whole batch instead of WriteDynamics2's text file
 * per simulation (tau.cu:3431-3469), for batches where text output would
 * dominate the run.  Little-endian layout: the 8 bytes "CTLSAMP1"; uint32 n,
 * ns, s_out, first_id; float64 t[ns]; uint32 species[s_out] (the sampled
 * species' indices); zero bytes up to a multiple of 16; then uint32
 * samples[n][ns][s_out] exactly as ctl_run returns them. */
ctl_status ctl_write_samples_binary(const ctl_model* m, const char* path, uint32_t n,
                                    const uint32_t* samples, uint32_t first_id);
/* Structured run report (the reference prints only "RUNNING TIME" under
 * verbose, kernel.cu:347): one JSON object with the batch size, the wall
 * seconds given, simulations and reaction firings per second, summed
 * steps / leaps / SSA steps / rejections, per-status counts, the algorithmic
 * HBM bytes per simulation and their rate, and the launch shape when
 * `launch` is not null.  Host code only. */
ctl_status ctl_write_run_report(const ctl_model* m, const char* path, uint32_t n, const ctl_sim_info* info,
                                double seconds, const ctl_launch_info* launch);

/* ---- fitness ------------------------------------------------------------- */
/* read_time_series (tau.cu:1056-1261): ts_rep, p_rep, ts_numtgt, tts_vector,
 * ts_matrix for a run of threads*blocks simulations. */
ctl_status ctl_target_load(const char* folder, const ctl_model* m, uint32_t threads,
                           uint32_t blocks, ctl_target** out);
void ctl_target_free(ctl_target* t);
ctl_status ctl_target_dims(const ctl_target* t, uint32_t* repetitions, uint32_t* p_rep,
                           uint32_t* target_quantities, uint32_t* experiments);
/* calculateFitness (tau.cu:3324-3408) on the GPU: fitness [threads*blocks]
 * (entries past threads*blocks/p_rep are 0). */
ctl_status ctl_fitness(ctl_model* m, const ctl_target* t, const ctl_run_cfg* cfg,
                       const uint32_t* samples, double* fitness);

/* calculateFitness (tau.cu:3324-3408) on device buffers: samples
 * [threads*blocks][ns][s_out], target [ns][experiments][repetitions][s_out],
 * experiment id per parameter set (uint8), fitness [threads*blocks/p_rep]. */
ctl_status ctl_fitness_device(const uint32_t* d_samples, uint32_t ns, uint32_t s_out,
                              const uint32_t* d_target, const uint8_t* d_experiment,
                              uint32_t experiments, uint32_t repetitions, uint32_t threads,
                              uint32_t blocks, uint32_t p_rep, double* d_fitness, void* stream);

/* ---- fitness mode without per-simulation samples ------------------------- */
/* Replaces the run + calculateFitness pair of the reference's fitness mode
 * (kernel.cu:347-423, 2phase_n-tau-leaping.cu:3324-3408) with a fused path:
 * the sweep adds every recorded sample into 64-bit integer sums per
 * parameter set instead of storing it (set of simulation gid =
 * (gid / (threads*p_rep)) * threads + gid % threads, the reference's layout);
 * the fitness then reads the sums.  Integer sums are exact, so the fitness
 * equals the one computed from stored samples bit for bit.
 * d_sums: [n / p_rep][ns][s_out] uint64, zeroed by the call. */
ctl_status ctl_run_device_sums(ctl_model* m, const ctl_run_cfg* cfg, uint32_t n, const int32_t* d_X0,
                               const float* d_c, uint32_t threads, uint32_t p_rep, uint64_t* d_sums,
                               ctl_sim_info* d_info, void* stream);
/* calculateFitness from the sums of ctl_run_device_sums (arguments as
 * ctl_fitness_device). */
ctl_status ctl_fitness_sums_device(const uint64_t* d_sums, uint32_t ns, uint32_t s_out,
                                   const uint32_t* d_target, const uint8_t* d_experiment,
                                   uint32_t experiments, uint32_t repetitions, uint32_t threads,
                                   uint32_t blocks, uint32_t p_rep, double* d_fitness, void* stream);
/* Host-buffer fitness mode: N = threads * blocks of the target, X0 [N][S],
 * c [N][R] -> fitness [N] (entries of the N / p_rep parameter sets first,
 * the rest 0, as ctl_fitness) and per-simulation records; CTL_ERR_STEP_LIMIT
 * if a simulation ended early. */
ctl_status ctl_fitness_run(ctl_model* m, const ctl_target* t, const ctl_run_cfg* cfg, const int32_t* X0,
                           const float* c, double* fitness, ctl_sim_info* info);

/* ---- surrogate MLP kernels (fitness-mode screening) ---------------------- */
/* No reference counterpart: the reference evaluates every candidate by full
 * simulation (kernel.cu:365-423).  These are the tcgen05 kernels that train
 * and run the screening surrogate; all pointers are device pointers. */
enum {
    CTL_EPI_ATOMIC_F32 = 0,  /* out_f32 += acc (split-K weight gradients)              */
    CTL_EPI_BIAS_SILU = 1,   /* z = acc + bias -> out_f32; silu(z) -> out_bf, out_bfT  */
    CTL_EPI_BIAS = 2,        /* out_f32 = acc + bias                                   */
    CTL_EPI_SILU_GRAD = 3,   /* acc * silu'(z_in) -> out_bf, out_bfT                    */
    CTL_EPI_F32 = 4          /* out_f32 = acc                                          */
};
typedef struct {
    const void* A;          /* BF16 [M][lda], K contiguous */
    const void* B;          /* BF16 [N][ldb], K contiguous */
    int32_t lda, ldb, M, N, K;  /* M % 128 == 0, N % 16 == 0 (N <= 256 or N % 256 == 0), K % 64 == 0 */
    int32_t epilogue;       /* CTL_EPI_* */
    int32_t splits;         /* split-K factor (CTL_EPI_ATOMIC_F32), 0 or 1 = none */
    const float* bias;      /* [N] */
    const float* z_in;      /* [M][ldz] */
    int32_t ldz;
    float* out_f32;         /* [M][ldo] */
    int32_t ldo;
    void* out_bf;           /* BF16 [M][ldob] */
    int32_t ldob;
    void* out_bfT;          /* BF16 [N][ldobT], optional */
    int32_t ldobT;
    unsigned* err;          /* device word, bit 0 raised if a bounded wait timed out */
} ctl_gemm_desc;
/* C = A . B^T on the 5th-generation tensor cores (tcgen05.mma, TMEM). */
ctl_status ctl_mlp_gemm(const ctl_gemm_desc* d, void* stream);
/* Gaussian NLL gradient w.r.t. y = [mean | log-variance | padding] (row
 * stride ldy >= 2S); dy BF16 [B][ldd], dyT BF16 [2S..][ldT]. */
ctl_status ctl_mlp_nll_grad(const float* y, int32_t ldy, const float* target, int32_t B, int32_t S,
                            void* dy, int32_t ldd, void* dyT, int32_t ldT, float* loss_sum, void* stream);
/* Column sums of a BF16 [B][N] matrix, added to g[N]. */
ctl_status ctl_mlp_colsum(const void* d, int32_t B, int32_t N, int32_t ld, float* g, void* stream);
/* One Adam step on FP32 weights [rows][cols]; refreshes BF16 W and W^T. */
ctl_status ctl_mlp_adam(float* w, const float* g, float* m1, float* m2, int32_t rows, int32_t cols,
                        float lr, float beta1, float beta2, float eps, int32_t step, float weight_decay,
                        void* w_bf16, void* wT_bf16, void* stream);

/* Fused surrogate screening (no reference counterpart: the reference scores
 * every candidate by full simulation, kernel.cu:365-423).  For each
 * candidate parameter set, runs the trained MLP at every sample instant and
 * returns the reference's fitness (calculateFitness,
 * 2phase_n-tau-leaping.cu:3324-3408) of the predicted ensemble mean against
 * the target: sum over instants and species of |target - mean| / target
 * (|target - mean| where the target is 0), divided by ns * S.  One kernel:
 * activations stay on chip, weights stream from ctl_mlp_pack's buffer. */
typedef struct {
    const float* theta;     /* [n_cand][n_par] log rate constants */
    int32_t n_par;          /* 1..63; network input = n_par scaled parameters + scaled t */
    uint32_t n_cand;
    const float* tvec;      /* [ns] sample instants */
    uint32_t ns;
    float t_end;            /* time scale of the input */
    const float* log_lo;    /* [n_par] prior box, maps theta to [-1, 1] */
    const float* log_hi;
    const float* y_mean;    /* [S] output de-standardisation: mean = y * y_std + y_mean */
    const float* y_std;
    int32_t S;              /* output species (2S <= out_w) */
    int32_t out_w;          /* output layer width (multiple of 16, <= 256) */
    const float* target;    /* [ns][S] */
    const void* wpack;      /* ctl_mlp_pack output (16-byte aligned) */
    const float* bias;      /* [4*256 + out_w]: the five layers' biases, concatenated (16-byte aligned) */
    double* fitness;        /* [n_cand] out */
    unsigned* err;          /* device word, bit 0 raised if a bounded wait timed out */
} ctl_screen_desc;
/* Bytes of the packed weights for an output width. */
size_t ctl_mlp_pack_bytes(int32_t out_w);
/* Packs BF16 weights W[0] [256][64], W[1..3] [256][256], W[4] [out_w][256]
 * (row strides ldw[l] elements) for ctl_mlp_screen. */
ctl_status ctl_mlp_pack(const void* const* W, const int32_t* ldw, int32_t out_w, void* wpack, void* stream);
ctl_status ctl_mlp_screen(const ctl_screen_desc* d, void* stream);
/* Checks the bounded waits of these kernels (no reference counterpart: the
 * reference has no waits that can give up): one warp waits on an mbarrier
 * that nothing arrives on, with nothing in flight, gives up after `limit`
 * polls (1 .. 2^24) and returns; *d_err then has bits 0 (the wait raised
 * its error) and 1 (the kernel saw the wait fail) set, which a caller reads
 * as CTL_ERR_TIMEOUT. */
ctl_status ctl_mlp_wait_check(unsigned* d_err, uint32_t limit, void* stream);

#ifdef __cplusplus
}
#endif
#endif
