/* ==========================================================================
 *  dynasor_b200.h -- C ABI of the B200 (sm_100a) sparse MTTKRP / CP-ALS
 *  engine (libdynasor_b200.so).
 *
 *  Plain C: opaque handles, raw host pointers and sizes, integer status
 *  codes.  No CUDA or torch types appear in any signature (CUDA streams are
 *  passed as void*).  Every function returns DGPU_OK (0) or a negative
 *  DGPU_ERR_* code; dgpu_last_error() gives a one-line description of the
 *  most recent failure on the calling thread.  Nothing here calls exit().
 *
 *  Data conventions are the reference's (include/dynasor_common.h:28-30,
 *  604-615, include/dynasor_linalg.h:8-17):
 *    * indices are 0-based uint32, values float32, COO as SoA
 *      (vals[nnz], idx[n][nnz]);
 *    * factor matrices are row-major I_n x Rp float32 with
 *      Rp = round_up(R, 16) and the padding columns zero;
 *    * the FLYCOO plan depends on the worker count `threads` exactly as the
 *      reference's plan depends on --threads, so a plan built here with
 *      threads=T produces the same slab permutation as the reference built
 *      with --threads T.
 *
 *  Threading: a plan is not thread-safe; its device work is ordered on one
 *  CUDA stream (its own, or one set with dgpu_plan_set_stream).  Work that
 *  the plan runs concurrently (the PingPong MTTKRP beside the remap, CP-ALS
 *  solve maps, host-buffer transfers) goes to the plan's internal streams,
 *  forked from and joined back into that stream before each call returns,
 *  so the stream sees every call as complete work in order.
 * ========================================================================== */
#ifndef DYNASOR_B200_H
#define DYNASOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGPU_MAX_MODES 8

/* ---- status codes --------------------------------------------------- */
#define DGPU_OK              0
#define DGPU_ERR_ARG        -1   /* bad argument / unsupported shape      */
#define DGPU_ERR_CUDA       -2   /* a CUDA runtime call failed            */
#define DGPU_ERR_NOMEM      -3   /* device or host allocation failed      */
#define DGPU_ERR_EMPTY      -4   /* tensor has no nonzeros / no modes     */
#define DGPU_ERR_INDEX      -5   /* an index is >= its mode size          */
#define DGPU_ERR_ORDER      -6   /* modes processed out of order          */
#define DGPU_ERR_IO         -7   /* file missing, truncated or malformed  */
#define DGPU_ERR_NOT_BUILT  -8   /* required plan state is missing        */
#define DGPU_ERR_DEVICE     -9   /* a kernel reported an internal fault   */

/* ---- layouts / kernels (values match the reference enums) ------------ */
#define DGPU_LAYOUT_PINGPONG 0   /* Layout::PingPong: remap every mode    */
#define DGPU_LAYOUT_NCOPY    1   /* Layout::NCopy: N pre-sorted copies    */
/* Layout::Morton (include/dynasor_common.h:133-155, src/dynasor_morton.cpp):
 * one 64-bit key per nonzero interleaving the mode indices (LSB-first round
 * robin, sum of ceil(log2 I_n) <= 64) plus the value, sorted by key; 12 bytes
 * per nonzero.  Only the all-modes pass runs on it (dgpu_mttkrp_all_modes,
 * dgpu_mttkrp_sweep, CP-ALS as Jacobi); dgpu_mttkrp_mode gives
 * DGPU_ERR_ARG.  dgpu_plan_morton reads the masks, keys and values. */
#define DGPU_LAYOUT_MORTON   4
/* Layout chosen from the device-memory budget like dyn_plan_storage
 * (src/dynasor_preprocess.cpp:951-1104): NCopy when it fits, else PingPong.
 * dgpu_plan_info.layout reports the choice.  (Not a reference enum value.) */
#define DGPU_LAYOUT_AUTO     16

#define DGPU_CP_GAUSS_SEIDEL 0   /* CpKernel::GaussSeidel                 */
#define DGPU_CP_JACOBI       1   /* CpKernel::Jacobi (all-modes pass)     */
#define DGPU_CP_AUTO         2   /* the compute plan's choice (the
                                    reference's --cp-kernel auto)        */

#define DGPU_PREC_FP32       0   /* FP32 gathers, FP32 accumulation       */
#define DGPU_PREC_BF16       1   /* BF16 gathers (FP32 master factors)    */

/* How the MTTKRP kernel accumulates Yhat rows. */
#define DGPU_ACCUM_AUTO      0   /* ROWRUN on fiber-sorted modes, else
                                    PRIVATE when the shard block fits     */
#define DGPU_ACCUM_ROWRUN    1   /* registers per row run + vector atomics
                                    at run ends (fast when rows are
                                    contiguous, i.e. fiber-sorted)       */
#define DGPU_ACCUM_PRIVATE   2   /* the super-shard's Yhat block in shared
                                    memory (any slab order; needs
                                    m_n * Rp * 4 <= ~200 KB)              */

typedef struct dgpu_plan dgpu_plan;   /* opaque */

/* Host COO tensor description (0-based indices). */
typedef struct {
    int             num_modes;
    uint64_t        nnz;
    const uint32_t* mode_size;    /* [num_modes]                         */
    const float*    vals;         /* [nnz]                               */
    const uint32_t* const* idx;   /* [num_modes][nnz]                    */
} dgpu_tensor_desc;

/* Plan options. */
typedef struct {
    int       threads;            /* reference worker count (>= 1)       */
    int       rank;               /* R (>= 1); Rp = round_up(R, 16)      */
    int       layout;             /* DGPU_LAYOUT_*                       */
    int       fiber;              /* 1: fiber-sort DenseFiber modes (the
                                     reference default); 0: the layout of
                                     DYN_FIBER_OFF=1                     */
    int       precision;          /* DGPU_PREC_*                         */
    int       device;             /* CUDA device ordinal                 */
    int       accum;              /* DGPU_ACCUM_*                        */
    const uint32_t* mn_target;    /* optional rows-per-shard override
                                     (NULL = pick like pick_mn)          */
} dgpu_plan_opts;

/* Per-mode plan facts (mirrors Tensor fields, include/dynasor_common.h:322-343). */
typedef struct {
    int       num_modes;
    uint64_t  nnz;
    int       rank;
    int       rank_padded;
    int       threads;
    uint32_t  mode_size[DGPU_MAX_MODES];
    uint32_t  mn[DGPU_MAX_MODES];               /* rows per super-shard   */
    int       mn_shift[DGPU_MAX_MODES];
    uint32_t  shards_per_mode[DGPU_MAX_MODES];
    int       kernel_class[DGPU_MAX_MODES];     /* 0 sparse,1 medium,2 dense */
    double    avg_fiber_len[DGPU_MAX_MODES];
    uint32_t  tiles[DGPU_MAX_MODES];            /* device work tiles      */
    int       next_mode;                        /* mode the slab is ready for */
    uint64_t  device_bytes;                     /* HBM held by the plan   */
    int       layout;                           /* DGPU_LAYOUT_PINGPONG / NCOPY in use */
} dgpu_plan_info;

/* CP-ALS options / result (mirror CpOptions / CpResult,
 * include/dynasor_cpals.h:82-114). */
typedef struct {
    int       max_iters;          /* default 50                           */
    double    tol;                /* stop when |fit_i - fit_{i-1}| < tol  */
    uint64_t  seed;               /* N(0,1) init seed (default 42)        */
    double    ridge;              /* relative ridge (default 1e-10)       */
    int       kernel;             /* DGPU_CP_* (DGPU_CP_AUTO: the compute
                                     plan's rule; default Gauss-Seidel)  */
    int       solve_fp64;         /* 1: FP64 Cholesky + solve (default)   */
    int       use_init;           /* 1: start from the uploaded factors   */
    int       verbose;            /* print the reference's [cpals] lines  */
    int       graphs;             /* 1: iterations after the first are
                                     captured once as a CUDA graph and
                                     replayed (default); 0: launch eagerly */
} dgpu_cp_options;

typedef struct {
    int       iters_done;
    double    final_fit;
    double    final_residual;
    double    tensor_norm;
    double    total_time_s;
    double    mttkrp_time_s;
    double    linalg_time_s;
} dgpu_cp_result;

/* ---- errors ----------------------------------------------------------- */
const char* dgpu_last_error(void);
int         dgpu_version(void);                   /* 0xMMmmpp             */
int         dgpu_device_count(int* count);

/* ---- plan (replaces build_flycoo: src/dynasor_preprocess.cpp:2013-2163) */
void dgpu_plan_opts_default(dgpu_plan_opts* opts);
int  dgpu_plan_create(const dgpu_tensor_desc* tensor, const dgpu_plan_opts* opts,
                      dgpu_plan** out);
int  dgpu_plan_destroy(dgpu_plan* plan);

/* ---- processed-tensor files (.dnp, src/dynasor_dnp.cpp) ---------------- */
/* layout_kind values of a .dnp header (src/dynasor_dnp.cpp:30-34) */
#define DGPU_DNP_MORTON      0
#define DGPU_DNP_NCOPY       1
#define DGPU_DNP_PINGPONG    2
#define DGPU_DNP_INPLACE     3

typedef struct {
    int       layout_kind;                      /* DGPU_DNP_*             */
    int       num_modes;
    uint64_t  nnz;
    uint32_t  mode_size[DGPU_MAX_MODES];
    int       num_threads;                      /* thread count the schedule
                                                   was built for          */
} dgpu_dnp_info;

/* Header of a .dnp file; host only, no device needed.  Replaces
 * load_dnp_header / load_dnp_num_threads / load_dnp_layout
 * (include/dynasor_dnp.h:127-140).  DGPU_ERR_IO for a missing file, bad
 * magic, version, value/index width, mode count, nnz or layout kind. */
int  dgpu_dnp_peek(const char* path, dgpu_dnp_info* info);

/* Plan from a .dnp file (runtime-only mode; replaces load_dnp_tensor,
 * include/dynasor_dnp.h:149-151, plus build_flycoo's work).  The file's
 * slab(s), shard tables and schedule are used as they are (no device sort);
 * the device checks index ranges, per-shard counts, shard order and, on
 * fiber-sorted NCopy copies, row order (DGPU_ERR_IO when one fails).
 * opts->threads must equal the file's thread count (DGPU_ERR_ARG, as the
 * reference rejects a mismatch); the file decides layout, rows per shard and
 * kernel classes (opts->layout and ->mn_target are ignored; so is
 * opts->fiber for NCopy files, whose copies say whether they are
 * fiber-sorted).  Morton files give a Morton plan: keys and values are
 * uploaded as they are and checked on the device (indices in range, keys
 * canonical and ascending).  InPlace files give DGPU_ERR_ARG. */
int  dgpu_plan_create_from_dnp(const char* path, const dgpu_plan_opts* opts,
                               dgpu_plan** plan);

/* Write the plan as a .dnp file (replaces save_dnp_tensor,
 * include/dynasor_dnp.h:121-123).  PingPong plans between sweeps (next mode
 * 0; DGPU_ERR_ORDER otherwise), NCopy and Morton plans at any time.  A plan built from
 * the same tensor with the same threads and layout writes the bytes the
 * reference writes after build_flycoo (NCopy: fiber-sorted copies carry
 * their CSR row pointers, as with --ncopy-csr-compact off).  Synchronises
 * the plan stream. */
int  dgpu_plan_save_dnp(const dgpu_plan* plan, const char* path);
int  dgpu_plan_get_info(const dgpu_plan* plan, dgpu_plan_info* info);
int  dgpu_plan_set_stream(dgpu_plan* plan, void* cuda_stream);
int  dgpu_plan_sync(dgpu_plan* plan);

/* Per-launch device timing (the reference only times phases with
 * omp_get_wtime, src/dynasor.cpp:393,538).  When enabled every kernel launch
 * is bracketed by CUDA events on the plan stream; dgpu_plan_get_timing
 * synchronises, folds the pending pairs into per-kind totals and copies
 * up to `max` records.  Kinds: "mttkrp", "part_hist", "part_scan",
 * "part_scatter", "zero", "linalg".  `bytes` is the algorithmic byte count
 * (each input read once, each output written once) summed over launches. */
typedef struct {
    char      name[24];
    uint64_t  launches;
    double    total_ms;
    double    bytes;
} dgpu_kernel_timing;
int dgpu_plan_set_timing(dgpu_plan* plan, int enable);
int dgpu_plan_get_timing(dgpu_plan* plan, dgpu_kernel_timing* out, int max,
                         int* count, int reset);

/* ---- autotuning (no single reference counterpart: the reference fixes its
 *      chunking at compile time; pick_mn, src/dynasor_preprocess.cpp:87-99,
 *      chooses only the rows per shard, and the plan keeps that choice) -----
 * Picks the plan's partition chunk sizes, LSD digit widths and MTTKRP grid
 * target by timing whole sweeps: coordinate descent over
 *   fiber_digit_bits {5,6,7,8}, sort_digit_bits {6,7,8}, chunks_per_sm
 *   {2,4,8}, seg_chunk_tiles {4,8,16} (PingPong plans; the fiber knobs only
 *   with fiber-sorted modes), mttkrp_ctas_per_sm {2,4,8} and the MTTKRP's
 *   row gathers (per-lane loads or TMA tile::gather4, 3- and 4-mode plans of
 *   Rp 16/32/64) (all layouts),
 * one warm-up and `sweeps` (1..50) timed sweeps per candidate, the fastest
 * kept.  No knob changes a slab permutation, and results change only by
 * FP32 summation order.  A PingPong plan must be between sweeps
 * (DGPU_ERR_ORDER otherwise); the sweeps it times advance its slab as any
 * sweep does (to the reference's slab after that many more sweeps), so tune
 * before work whose slab order matters.  Cached CP-ALS graphs of the plan
 * are recaptured afterwards.  Morton plans give DGPU_ERR_ARG.  Synchronises. */
typedef struct {
    int       fiber_digit_bits;      /* bits per LSD pass of the fiber sort */
    int       sort_digit_bits;       /* bits per LSD pass of the remap      */
    int       chunks_per_sm;         /* remap partition chunks per SM       */
    int       seg_chunk_tiles;       /* fiber partition: 4096-nnz tiles per chunk */
    int       mttkrp_ctas_per_sm;    /* MTTKRP tile split target            */
    int       mttkrp_gather;         /* 1: rows by TMA tile::gather4        */
    int       candidates;            /* configurations timed                */
    double    default_ms;            /* ms per sweep before tuning          */
    double    tuned_ms;              /* ms per sweep with the chosen values */
} dgpu_tune_result;
int dgpu_plan_autotune(dgpu_plan* plan, int sweeps, dgpu_tune_result* out);

/* Plan tables (src/dynasor_preprocess.cpp:291-463): shard ranges of mode n
 * (K entries each), and the LPT schedule as per-worker counts plus the
 * concatenated shard lists.  *n_listed receives the number of shards. */
int dgpu_plan_shards(const dgpu_plan* plan, int n, uint64_t* begin, uint64_t* end);
int dgpu_plan_schedule(const dgpu_plan* plan, int n, uint32_t* counts,
                       uint32_t* flat, uint32_t* n_listed);

/* ---- factors ---------------------------------------------------------- */
/* Y[n] <- host I_n x Rp row-major FP32 (replaces FactorMatrices::Y,
 * include/dynasor_common.h:604-615). */
int dgpu_upload_factor(dgpu_plan* plan, int n, const float* Y);
int dgpu_download_factor(dgpu_plan* plan, int n, float* Y);
int dgpu_download_yhat(dgpu_plan* plan, int n, float* Yhat);
int dgpu_download_lambda(dgpu_plan* plan, float* lambda);
/* Device pointers of Y[n] / Yhat[n] (I_n x Rp FP32), for zero-copy use. */
int dgpu_factor_device_ptr(dgpu_plan* plan, int n, void** Y, void** Yhat);

/* ---- MTTKRP (replaces SpmttkrpSweep::process, src/dynasor.cpp:352-539,
 *      and dynasor_process_shard, src/dynasor_kernel.cpp:289-338) ------- */
/* Mode n MTTKRP into Yhat[n]; under PingPong also remaps the slab for mode
 * (n+1) % N on the device.  Modes must be called in order 0,1,..,N-1,0,..
 * (DGPU_ERR_ORDER otherwise).  Asynchronous on the plan stream. */
int dgpu_mttkrp_mode(dgpu_plan* plan, int n);
/* All N modes in order (spmttkrp_dynasor, src/dynasor.cpp:545-559). */
int dgpu_mttkrp_sweep(dgpu_plan* plan);
/* All-modes single pass from one factor snapshot (Jacobi;
 * spmttkrp_all_modes_dynasor, src/dynasor.cpp:592-817). */
int dgpu_mttkrp_all_modes(dgpu_plan* plan);
/* Host-buffer convenience: upload Y[0..N-1], one sweep, download
 * Yhat[0..N-1] (spmttkrp_dynasor on host factor matrices).  Transfers run
 * on a second stream overlapping the mode passes (Y[0] while mode 0 runs,
 * Yhat[n] while the later modes run); pinned host buffers make that
 * overlap real.  Returns when all copies are done; *secs = device seconds
 * of the mode passes. */
int dgpu_mttkrp_sweep_host(dgpu_plan* plan, const float* const* Y,
                           float* const* Yhat, double* secs);

/* Current slab as the next mode's kernel will read it (bit-exact layout
 * checks against the reference's Tensor after process(n)).  A Morton plan
 * gives its nonzeros in key order with the indices decoded from the keys. */
int dgpu_download_slab(dgpu_plan* plan, float* vals, uint32_t* const* idx);
/* NCopy copy k (layout NCopy only). */
int dgpu_download_copy(dgpu_plan* plan, int k, float* vals, uint32_t* const* idx);
/* Morton layout state (T.morton_mask / morton_bits / morton_keys /
 * morton_vals after build_morton_layout, src/dynasor_morton.cpp:143-352):
 * mask[n] and bits[n] for n < num_modes, and, when keys / vals are not
 * NULL, the nnz sorted keys and their values.  DGPU_ERR_NOT_BUILT unless
 * the plan's layout is DGPU_LAYOUT_MORTON.  Synchronises the plan stream. */
int dgpu_plan_morton(dgpu_plan* plan, uint64_t* mask, uint8_t* bits, uint64_t* keys,
                     float* vals);

/* ---- CP-ALS (replaces cpals, src/dynasor_cpals.cpp:120-396) ---------- */
void dgpu_cp_options_default(dgpu_cp_options* opt);
/* fit_history receives one FP64 fit per iteration (max_iters entries). */
int  dgpu_cpals(dgpu_plan* plan, const dgpu_cp_options* opt,
                dgpu_cp_result* res, double* fit_history);

/* The reference's seeded N(0,1) initial factor of mode n (init_random_factors,
 * src/dynasor_cpals.cpp:42-69): rows x Rp row-major host buffer, padding
 * zero; the draws dgpu_cpals starts from.  Host only, no device needed. */
int  dgpu_init_factor(uint64_t seed, int n, uint32_t rows, int R, int Rp, float* Y);

/* K random-restart CP-ALS runs in one plan (no single reference function:
 * the reference runs cpals, src/dynasor_cpals.cpp:120-396, once per seed).
 * The plan's rank is restarts * Re (Re <= 64); restart k uses columns
 * [k*Re, (k+1)*Re) of every factor, starts from the reference's N(0,1)
 * initialisation with seed opt->seed + k (unless opt->use_init), and has its
 * own fit and stop rule; a converged restart is frozen while the others
 * continue.  One MTTKRP sweep serves all restarts.  res[restarts];
 * fit_history (may be NULL) receives restarts x max_iters fits (row k =
 * restart k, zero after its last iteration).  total_time_s is the batch's
 * wall time; mttkrp_time_s and linalg_time_s are 0 (not split). */
int  dgpu_cpals_multistart(dgpu_plan* plan, int restarts, const dgpu_cp_options* opt,
                           dgpu_cp_result* res, double* fit_history);
/* Independent CP-ALS runs on `count` plans (one per tensor, same device),
 * each as dgpu_cpals would run it; after every plan's first iteration the
 * remaining iterations of all plans run as parallel device-side loops of
 * one CUDA graph launch (no reference counterpart: the reference decomposes
 * one tensor per process).  res[count]; fit_history (may be NULL) receives
 * count x max_iters fits, row k for plans[k]. */
int  dgpu_cpals_batch(dgpu_plan* const* plans, int count, const dgpu_cp_options* opt,
                      dgpu_cp_result* res, double* fit_history);

/* ---- compute plan (replaces ComputePlan, dyn_build_compute_plan and
 *      dyn_print_compute_plan: include/dynasor_common.h:244-320,
 *      src/dynasor_preprocess.cpp:1179-1399) ---------------------------------
 * The run-time decisions of a plan in one record: the CP-ALS kernel
 * (Jacobi or Gauss-Seidel, chosen by the reference's rule: Morton layout ->
 * Jacobi; nnz < 1M -> Gauss-Seidel; N == 3 and Rp >= 64, or Rp >= 128 ->
 * Gauss-Seidel; the reference's per-thread all-modes output copies
 * (threads x sum_n I_n*Rp*4, each rounded to 64 B) >= min(MemAvailable/4,
 * 8 GiB) -> Gauss-Seidel; else Jacobi), the reference's per-mode kernel
 * class, and what this engine runs per mode (accumulation scheme, rank
 * tile).  kernel_cli takes the reference's keywords ("auto", "jacobi",
 * "all-modes", "js", "gs", "gauss-seidel", "per-mode", ...; NULL = auto);
 * the DYN_CP_KERNEL environment variable overrides it as in the reference. */
#define DGPU_IMPL_ELEMENT    0   /* KernelImpl::Element                   */
#define DGPU_IMPL_FIBER      1   /* KernelImpl::Fiber                     */
#define DGPU_IMPL_FIBERCSR   2   /* KernelImpl::FiberCSR                  */

/* Tensor facts the decision needs (no device involved). */
typedef struct {
    int       num_modes;
    uint64_t  nnz;
    uint32_t  mode_size[DGPU_MAX_MODES];
    int       rank_padded;
    int       threads;
    int       layout;                           /* DGPU_LAYOUT_PINGPONG/NCOPY/MORTON */
    int       fiber;                            /* NCopy copies fiber-sorted  */
    int       kernel_class[DGPU_MAX_MODES];     /* 0 sparse, 1 medium, 2 dense */
    double    avg_fiber_len[DGPU_MAX_MODES];
    uint64_t  host_avail_bytes;                 /* 0: MemAvailable of /proc/meminfo */
} dgpu_compute_plan_input;

typedef struct {
    int       layout;                           /* DGPU_LAYOUT_* of the plan  */
    int       kernel;                           /* DGPU_CP_GAUSS_SEIDEL / JACOBI */
    char      kernel_reason[48];
    char      kernel_source[16];                /* auto | cli-kernel | env-kernel */
    int       per_mode[DGPU_MAX_MODES];         /* DGPU_IMPL_* (reference class) */
    int       accum[DGPU_MAX_MODES];            /* DGPU_ACCUM_ROWRUN / PRIVATE used
                                                   here (0: all-modes pass only) */
    int       rank_tile[DGPU_MAX_MODES];        /* columns per slab pass
                                                   (0: tuned at first use) */
    int       precision;                        /* DGPU_PREC_*                */
    int       num_modes;
    int       rank_padded;
    int       threads;
    uint64_t  ofibs_bytes;                      /* reference all-modes copies  */
    uint64_t  factor_bytes;                     /* sum_n I_n * Rp * 4 * 2      */
    uint64_t  budget_bytes;                     /* min(MemAvailable/4, 8 GiB)  */
    uint64_t  device_bytes;                     /* HBM held by the plan        */
} dgpu_compute_plan;

/* The decision from tensor facts alone (host only; device fields zero). */
int dgpu_compute_plan_decide(const dgpu_compute_plan_input* in, const char* kernel_cli,
                             dgpu_compute_plan* out);
/* The decision for a built plan, with its device facts filled in. */
int dgpu_build_compute_plan(const dgpu_plan* plan, const char* kernel_cli,
                            dgpu_compute_plan* out);
/* The plan banner (one "<prefix> key : value" line per row, like
 * dyn_print_compute_plan) into buf; DGPU_ERR_ARG when cap is too small. */
int dgpu_format_compute_plan(const dgpu_compute_plan* cp, const char* prefix, char* buf,
                             size_t cap);

/* ---- small dense kernels (replace la::*, include/dynasor_linalg.h:33-127),
 *      device pointers, FP32 row-major with leading dimension Rp --------- */
int dgpu_la_gram(void* stream, const float* Y, uint64_t rows, int R, int Rp, float* G);
int dgpu_tensor_norm_sq(dgpu_plan* plan, double* norm_sq);

/* ---- CP-OPT forward / adjoint (no reference counterpart: the gradient
 *      of 0.5*||X - M||^2 over the nonzeros, built from MTTKRP) -------- */
/* model[i] = sum_r prod_n Y[n][idx_n(i), r] at every nonzero, in the
 * current slab order (FP32 out). */
int dgpu_model_values(dgpu_plan* plan, float* model_host);
/* grad[n] = -(MTTKRP_n(X) - Y[n] * Hadamard_{m!=n}(Y[m]^T Y[m])), the
 * gradient of 0.5*||X - M||_F^2 w.r.t. Y[n] for the dense CP model M,
 * written to host I_n x Rp FP32 buffers. */
int dgpu_cpopt_gradient(dgpu_plan* plan, float* const* grad_host);

/* ---- allocation-free stable shard partition (no counterpart in the
 *      reference: an addition for callers that may not allocate device
 *      memory, e.g. code whose device memory is owned by a host framework's
 *      pool, or latency-critical paths where cudaMalloc's device-wide
 *      synchronisation is not allowed) ------------------------------------
 * Stable counting sort of a device SoA slab, taken in slab order, by key =
 * idx[key_mode][i] >> key_shift (< num_buckets <= 2048), from
 * (vals_in, idx_in[]) into (vals_out, idx_out[]) -- the partition the remap
 * and the initial mode-0 shard order use.  idx_in/idx_out are host arrays
 * of num_modes device pointers.  Allocates nothing: its scratch is one fixed
 * 16 MiB device array that every GPU loading the library holds until exit;
 * requests needing more than 2,095,104 counters (num_buckets *
 * ceil(nnz / 4096)) are rejected with DGPU_ERR_ARG.  Calls share that
 * array, so calls whose device work overlaps race; the first call on a
 * device resolves the array's address and should come before any stream
 * capture, and that address is kept (cudaDeviceReset on the device after
 * the first call is not supported).  Waits for `stream` before returning,
 * so a call on a stream that is being captured gives DGPU_ERR_ARG; a key
 * >= num_buckets yields DGPU_ERR_INDEX. */
int dgpu_sort_slab_noalloc(void* stream, int num_modes, uint64_t nnz,
                           const float* vals_in, const uint32_t* const* idx_in,
                           float* vals_out, uint32_t* const* idx_out,
                           int key_mode, int key_shift, uint32_t num_buckets);

/* ---- host loaders (replace load_coo_tensor / save_dnb_tensor /
 *      dump_factor_matrix_bin, src/dynasor_io.cpp:576-1348) ---------------- */
/* A host COO tensor owned by the library (free with dgpu_coo_free). */
typedef struct {
    int       num_modes;
    uint64_t  nnz;
    uint32_t  mode_size[DGPU_MAX_MODES];
    float*    vals;
    uint32_t* idx[DGPU_MAX_MODES];
} dgpu_coo;

/* <path>.dnb when fresh, else parse <path> (.tns) and, when use_cache,
 * write <path>.dnb (src/dynasor_io.cpp:1184-1261). */
int  dgpu_load_coo_tensor(const char* path, int use_cache, dgpu_coo* out);
int  dgpu_load_tns(const char* path, dgpu_coo* out);        /* :576-745  */
int  dgpu_load_dnb(const char* path, dgpu_coo* out);        /* :805-850  */
int  dgpu_save_dnb(const char* path, const dgpu_coo* t);    /* :854-893  */
void dgpu_coo_free(dgpu_coo* t);
/* DYFM dump of an I x rank_padded factor, padding stripped (:1287-1348). */
int  dgpu_dump_factor_bin(const char* path, const float* data, uint32_t rows,
                          int rank, int rank_padded);

#ifdef __cplusplus
}
#endif
#endif /* DYNASOR_B200_H */
