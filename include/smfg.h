/*
 * smfg.h -- C ABI of the B200 numeric phase for smf (sparse symmetric
 * multifrontal LDL^T / Cholesky). Plain pointers and sizes only.
 *
 * The engine takes smf's symbolic analysis as is (the AnalysisKeep arrays,
 * solver/include/smf/analysis.hpp:25-144) and replaces the numeric phase
 * behind smf::Solver::factor / solve (solver/include/smf/solver.hpp:78-114),
 * i.e. the body of multifrontal_factor_serial
 * (solver/src/multifrontal_serial.cpp:1105) and of solve_core's forward /
 * diagonal / backward passes (solver/src/solve.cpp:858-1075), on one GPU.
 *
 * All indices are 0-based int32; dense blocks are column-major.
 *
 * Calls taking device pointers run on the plan's own stream after the work
 * the calling thread has queued on the legacy default stream (where a
 * caller's copies or torch kernels wrote the inputs), and return once their
 * own work is done.
 */
#ifndef SMFG_H
#define SMFG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SMFG_API __attribute__((visibility("default")))
#else
#define SMFG_API
#endif

#define SMFG_ABI_VERSION 1

/* Status codes. 0..5 are smf_c.h's SMF_OK .. SMF_ERR_INEXACT_INERTIA
 * (solver/include/smf/smf_c.h:83-88); the rest are specific to the device. */
#define SMFG_OK 0
#define SMFG_ERR_INVALID_ARG 1
#define SMFG_ERR_SINGULAR 2       /* zero pivots, or not positive definite (SPD path) */
#define SMFG_ERR_INTERNAL 3
#define SMFG_ERR_WRONG_INERTIA 4  /* more negative pivots than max_negative_pivots */
#define SMFG_ERR_INEXACT_INERTIA 5
#define SMFG_ERR_CUDA 10          /* a CUDA runtime call failed */
#define SMFG_ERR_NO_DEVICE 11
#define SMFG_ERR_NONFINITE 12     /* non-finite input values (smf ErrorCode::IllegalValue) */
#define SMFG_ERR_ARENA 13         /* device arena too small (delays); retried internally */
#define SMFG_ERR_TIMEOUT 14       /* a bounded device wait gave up */

/* Factor status (smf::FactorStatus, solver/include/smf/types.hpp:230-238). */
#define SMFG_FACTOR_SUCCESS 0
#define SMFG_FACTOR_NOT_POSDEF 1
#define SMFG_FACTOR_SINGULAR 2
#define SMFG_FACTOR_MAX_PIVOT_DELAYS 3  /* stopped at the work limit (smfg_control_t.work_limit) */
#define SMFG_FACTOR_INERTIA_EXCEEDED 4  /* stopped once the negative pivots passed max_negative_pivots */

/* Solve jobs (smf::SolveJob / SMF_SOLVE_*). */
#define SMFG_SOLVE_FULL 0
#define SMFG_SOLVE_FORWARD 1
#define SMFG_SOLVE_DIAGONAL 2
#define SMFG_SOLVE_BACKWARD 3

/* Schur-update precision of large fronts. */
#define SMFG_PREC_FP64 0          /* plain FP64, the reference's arithmetic */
#define SMFG_PREC_MIXED 1         /* tensor-core reduced precision where the selector allows */

/* The analysis the numeric phase consumes: the AnalysisKeep arrays of smf
 * (analysis.hpp:25-144) that multifrontal_factor_serial reads. Supernodes are
 * numbered in postorder; children are listed in descending postorder (the
 * order the reference's LIFO contribution stack consumes them); each front's
 * rows are sorted ascending, its first (sn_end - sn_start) rows being its
 * pivots. The permuted lower pattern (perm_col_ptr / perm_row_idx, new
 * numbering, rows >= column) is where the values are placed. */
typedef struct {
  int n;
  int nsn;
  const int *perm;          /* perm[new] = old, n */
  const int *sn_start;      /* nsn */
  const int *sn_end;        /* nsn */
  const int *sn_parent;     /* nsn, -1 at roots */
  const int *child_ptr;     /* nsn + 1 */
  const int *child_idx;     /* child_ptr[nsn] */
  const int *front_row_ptr; /* nsn + 1 */
  const int *front_row_idx; /* front_row_ptr[nsn] */
  const int *postorder;     /* nsn */
  const int *perm_col_ptr;  /* n + 1 */
  const int *perm_row_idx;  /* perm_col_ptr[n] */
  /* Value placement: input entry k (the caller's order, nnz_in entries) goes
   * to cleaned slot orig_to_clean[k] (-1 = dropped; duplicates summed in
   * input order), cleaned slot c to permuted slot clean_to_perm[c]; the
   * cleaned pattern (clean_col_ptr / clean_row_idx, original numbering)
   * gives each slot's row and column for the scaling S A S.
   * AnalysisKeep::orig_to_clean_idx, orig_to_perm_idx, cleaned. */
  int64_t nnz_in;
  const int *orig_to_clean; /* nnz_in */
  const int *clean_to_perm; /* clean_col_ptr[n] */
  const int *clean_col_ptr; /* n + 1 */
  const int *clean_row_idx; /* clean_col_ptr[n] */
} smfg_analysis_t;

typedef struct {
  int abi_version;        /* SMFG_ABI_VERSION */
  int posdef;             /* 1: Cholesky path (smf's SPD factor_posdef) */
  double u;               /* threshold pivoting parameter (Control::pivot_u) */
  double small_pivot;     /* zero-pivot threshold (Control::small_pivot) */
  int nb;                 /* panel width (Control::indef_panel_size, 16) */
  int blocked_min_front;  /* blocked kernel from this many rows (96) */
  int precision;          /* SMFG_PREC_* */
  int max_negative_pivots;/* < 0: off (Control::max_negative_pivots). Indefinite: the
                             factorization stops after the tree level at which the negative
                             pivots so far pass it (the rest skipped, SMFG_ERR_WRONG_INERTIA,
                             SMFG_FACTOR_INERTIA_EXCEEDED, partial counts; the factor is
                             unusable), multifrontal_serial.cpp:1619-1628 */
  const double *scale;    /* optional S (length n, original numbering), NULL = none */
  int profile;            /* 1: time the large-front update kernels (info.reserved_d[0..1]) */
  /* SMFG_PREC_MIXED: large fronts of at least mixed_min_front rows (0: 1024
   * for an SPD factorization, 384 for an indefinite one)
   * that smfg_set_front_precision allows are factored in outer blocks of
   * mixed_block pivots (0: 256; a multiple of 64): the threshold-pivoting
   * panels stay FP64 and the columns past each block get one tensor-core
   * update of kind mixed_kind (SMFG_TC_TF32X3 or SMFG_TC_BF16X3). */
  int mixed_block;
  int mixed_kind;
  int mixed_min_front;
  int panel_team;         /* CTAs per indefinite large front's pivoting (1, 2, 4, 8, 16); 0: by front size */
  /* 1: replay the factorization as one CUDA graph. The first call with a
   * given configuration (control, precision mask, value pointer) factors
   * normally and captures the launch sequence; later calls with the same
   * configuration replay it (the refactor of an interior-point iteration).
   * A replay that finds a front needing more pivoting steps than captured,
   * or an arena too small, falls back to the normal path. */
  int graph;
  /* Dense kernel of the indefinite fronts: fronts of at least aptp_min_rows
   * realized rows take a posteriori threshold pivoting in 256-column tiles,
   * then the threshold kernel on the columns it failed -- smf's
   * deterministic mode (multifrontal_serial.cpp:796-821, kTopTileMinFront =
   * 512, parallel/thread_plan.hpp:43), the default (512). 0: the threshold
   * kernel on every front (smf's one-thread default mode). Plans whose
   * indefinite factorizations reach such fronts are not captured as a graph
   * (graph = 1 then factors without capture). */
  int aptp_min_rows;
  int reserved_i[1];
  /* Indefinite: >= 0 stops the factorization after the tree level at which
   * the front work so far (sum over fronts of fully summed columns x
   * rows^2) passes floor(work_limit) -- the scale-on-delay rescue's limit
   * (multifrontal_serial.cpp:660-671): status SMFG_OK, factor_status
   * SMFG_FACTOR_MAX_PIVOT_DELAYS, no usable factor. < 0: off. */
  double work_limit;
  double reserved_d[7];
} smfg_control_t;

typedef struct {
  int status;             /* SMFG_OK or an error code */
  int factor_status;      /* SMFG_FACTOR_* */
  int num_pos, num_neg, num_zero;
  int delayed_pivots;
  int two_by_two_pivots;
  int max_front;
  int64_t factor_entries; /* sum over fronts of f * p */
  double flops;           /* smf's actual_flops count */
  double max_abs;         /* max |S A S| */
  double factor_ms;       /* device time of the last factor */
  double solve_ms;        /* device time of the last solve */
  int levels;
  int kernel_launches;    /* kernels launched by the last call */
  int mixed_fronts;       /* fronts whose trailing updates ran on the tensor cores */
  int reserved_i[7];      /* [0] profiled FP64 update launches, [1] tensor-core update passes,
                             [2] deferred front updates, [3] those of at most 2 pivots,
                             [4] columns the APTP sweeps failed (Info::aptp_failed_columns),
                             [5] fronts swept by APTP */
  double reserved_d[8];   /* [0] profiled FP64 update ms (deferred + Schur), [1] FP64 update
                             flops, [2] arena bytes, [3] tensor-core update flops (2 per
                             multiply-add), [4] profiled tensor-core update ms (split + product
                             kernels), [5] profiled large-front pivoting panel ms, [6] deferred
                             update bytes (each element read and written once), [7] profiled
                             Schur update ms (part of [0]) */
} smfg_info_t;

typedef struct smfg_plan_s *smfg_plan_t;

SMFG_API int smfg_abi_version(void);
SMFG_API void smfg_default_control(smfg_control_t *ctrl);

/* Device plan from an analysis (host arrays). Replaces the per-analysis
 * set-up of multifrontal_factor_serial (multifrontal_serial.cpp:1105-1300):
 * level sets of the assembly tree, child -> parent row maps, value-placement
 * maps, arena sizes. device < 0: the current device. */
SMFG_API int smfg_plan_create(const smfg_analysis_t *a, int device, smfg_plan_t *out);
SMFG_API void smfg_plan_destroy(smfg_plan_t *plan);

/* Numeric factorization of new values (the caller's entry order, nnz_in
 * host doubles) -- Solver::factor(ak, values, ...) (solver.hpp:88-90). */
SMFG_API int smfg_factor(smfg_plan_t plan, const double *values, const smfg_control_t *ctrl,
                         smfg_info_t *info);
/* The same with the values already in device memory. */
SMFG_API int smfg_factor_device(smfg_plan_t plan, const double *d_values,
                                const smfg_control_t *ctrl, smfg_info_t *info);

/* Solve in place: b is n x nrhs column-major with leading dimension ldb,
 * host memory -- Solver::solve (solver.hpp:101-114). */
SMFG_API int smfg_solve(smfg_plan_t plan, double *b, int nrhs, int ldb, int job, smfg_info_t *info);
/* The same with b in device memory. */
SMFG_API int smfg_solve_device(smfg_plan_t plan, double *d_b, int nrhs, int ldb, int job,
                               smfg_info_t *info);

/* Inertia of the last factorization (smf_inertia, smf_c.h:175). */
SMFG_API int smfg_inertia(smfg_plan_t plan, int *pos, int *neg, int *zero);

/* Per-front precision choice for SMFG_PREC_MIXED factorizations (a
 * learned selector's output, or the FP64 fallback after a misjudged
 * front): mask[s] = 1 lets supernode s take tensor-core trailing updates
 * (large fronts only), 0 keeps it in FP64. NULL: every large front may.
 * Kept for later factorizations until changed. */
SMFG_API int smfg_set_front_precision(smfg_plan_t plan, const int8_t *mask);

/* Tuned team sizes of the indefinite large-front pivoting (an autotuner's
 * choice; no reference counterpart): teams[b] CTAs (1, 2, 4, 8, 16; 0 = the
 * built-in rule) for levels whose largest front has [384, 768), [768,
 * 1536), [1536, 3072), >= 3072 symbolic rows (b = 0..3). NULL resets.
 * smfg_control_t.panel_team, when set, overrides the table. Kept for later
 * factorizations. */
SMFG_API int smfg_set_panel_teams(smfg_plan_t plan, const int *teams);

/* Per-front export of the last factor, in the FactorKeep layout
 * (factor_posdef.hpp:43-220): for supernode s, f[s] realized rows, p[s]
 * stored pivots, its L block (f x p, leading dimension f, D inline for the
 * indefinite path) copied to blocks + blk_off[s] (packed in supernode
 * order), rows (pivot order) to rows + row_off[s], pivot tags (1, 2, -1, 0)
 * to tags + tag_off (sum of earlier p). Sizes from smfg_factor_sizes. */
SMFG_API int smfg_factor_sizes(smfg_plan_t plan, int64_t *block_entries, int64_t *row_entries);
SMFG_API int smfg_factor_export(smfg_plan_t plan, int *f, int *p, int64_t *blk_off, double *blocks,
                                int64_t *row_off, int *rows, int8_t *tags);

/* Per-front counts of the last factorization: stats[5 s .. 5 s + 4] =
 * positive, negative and zero pivots, 2x2 pivots, delayed columns passed to
 * the parent (the per-front parts of Info's counts). Lets a caller that
 * factors many independent systems as one forest read each system's
 * inertia. */
SMFG_API int smfg_front_stats(smfg_plan_t plan, int *stats);

/* Residual r = b - A x and backward errors against the factored values
 * (refinement.cpp:39-130; compensated FP64 on the device). Host arrays. */
SMFG_API int smfg_residual(smfg_plan_t plan, const double *b, const double *x, int nrhs, double *r,
                           double *eta_inf, double *omega);

/* smfg_residual for callers that cannot allocate memory. Not a counterpart
 * of any reference interface: smf has no such entry point. Some callers
 * must not allocate device memory once they are running: a real-time
 * controller that reserves everything at start-up (cudaMalloc can block for
 * an unbounded time and may synchronize the device), or a host program whose
 * memory is owned by its own pool allocator and already committed to it, so
 * that an extra cudaMalloc fails for want of memory. smfg_residual allocates
 * its scratch on every call; this variant takes device buffers (b, x and r:
 * n x nrhs, leading dimension n; r may be NULL) and works in a fixed scratch
 * array compiled into the library, sized for n <= SMFG_NOALLOC_MAX_N
 * (262,144: about 6 MB that every GPU which loads the library holds until
 * the process exits, whether or not this entry point is ever called). A
 * larger plan is rejected with SMFG_ERR_INVALID_ARG, a plan that has not been
 * factored with SMFG_ERR_SINGULAR. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture. Every call shares the one array and the maxima
 * in it are cleared at the start of each column, but calls that overlap on
 * the GPU (from other threads or streams) race on it: serialize them. The
 * call waits for its kernels (it synchronizes the plan's stream) and copies
 * the error maxima back to the host to return them. */
#define SMFG_NOALLOC_MAX_N 262144
SMFG_API int smfg_residual_noalloc(smfg_plan_t plan, const double *d_b, const double *d_x, double *d_r,
                                   int nrhs, double *eta_inf, double *omega);

/* Kernel self-benchmark (no reference counterpart): the streamed deferred
 * update on one synthetic front of f rows, ne eligible columns, a pending
 * panel of k <= 16 pivots; best device time of reps launches (ms), the
 * update's algorithmic bytes, and the entries whose bits differ from the
 * tiled kernel's result (0 expected). Allocates 3 (f^2 + 16 f) doubles. */
/* Kernel self-test (no reference counterpart as an entry point): the APTP
 * front kernel that factors every indefinite front of at least 512 rows
 * (deterministic mode's kernel, solver/src/ldlt_aptp.cpp:739) on one dense
 * front in device memory: d_F f x f column-major (lower triangle), its first
 * ne columns eligible, d_rows / d_tags (f) permuted and tagged in place,
 * threshold u, zero-pivot value small. out[0..4] = pivots eliminated,
 * columns failed, positive, negative, zero pivots. The failed columns are
 * left behind the pivots with their Schur complement current (the caller's
 * threshold kernel takes them next). Allocates its scratch. */
SMFG_API int smfg_aptp_front_dense(double *d_F, int f, int ne, int *d_rows, int8_t *d_tags, double u, double small,
                                   int64_t *out);
SMFG_API int smfg_kernel_bench_defer(int f, int ne, int k, int reps, double *ms, double *bytes,
                                     long long *mismatches);

/* Iterative refinement (classical, refinement.cpp:316-413) of x for b, host
 * arrays (n x nrhs, leading dimension n): at most max_steps solves, stopping
 * at eta_inf <= 1e-10 and omega <= omega_target. */
SMFG_API int smfg_refine(smfg_plan_t plan, const double *b, double *x, int nrhs, int max_steps,
                         double omega_target, double *eta_inf, double *omega, int *steps);

/* Refinement methods (smf::RefineMethod, solver/include/smf/types.hpp:160-170):
 * classical x += M^-1 r; right-preconditioned FGMRES(restart) with the
 * factor as preconditioner (refinement.cpp:451-643); auto = classical,
 * escalating to FGMRES when a step contracts the gate measure by less than
 * 0.5 (on a factor with mixed-precision fronts auto is FGMRES). Gate: eta_inf <= 1e-10 and omega <= omega_target; at most max_iters
 * solves in all; x is left at the best iterate. restart <= 0: 20. */
#define SMFG_REFINE_CLASSICAL 0
#define SMFG_REFINE_FGMRES 1
#define SMFG_REFINE_AUTO 2
SMFG_API int smfg_refine_method(smfg_plan_t plan, const double *b, double *x, int nrhs, int method,
                                int max_iters, int restart, double omega_target, double *eta_inf,
                                double *omega, int *iters);
/* The same with b and x in device memory (n x nrhs, leading dimension n). */
SMFG_API int smfg_refine_device(smfg_plan_t plan, const double *d_b, double *d_x, int nrhs, int method,
                                int max_iters, int restart, double omega_target, double *eta_inf,
                                double *omega, int *iters);

/* Device times (CUDA events on the plan's stream) of the last factor, solve
 * and refinement; a refinement's time includes its waits for the host's
 * small Hessenberg work between iterations. */
SMFG_API int smfg_last_times(smfg_plan_t plan, double *factor_ms, double *solve_ms, double *refine_ms);

/* Symmetric max-product matching scaling (host code): the scaling smf
 * applies before an indefinite factorization when matching scaling is on
 * (solver/src/scaling_matching.cpp): a minimum-cost perfect matching on
 * c_ij = log max_k |a_kj| - log |a_ij| (MC64 job 5) and scale[i] =
 * exp((u_i + v_i) / 2) / sqrt(max_k |a_ki|) from its dual potentials, so
 * that |s_i a_ij s_j| <= 1 with equality on the matched entries. Input:
 * lower CSC (original numbering); scale: n doubles, to pass as
 * smfg_control_t.scale. *unmatched: columns left without a match
 * (structurally singular). SMFG_ERR_SINGULAR for an all-zero row. */
SMFG_API int smfg_matching_scale(int n, const int *col_ptr, const int *row_idx, const double *values,
                                 double *scale, int *unmatched);

/* The learned per-front precision selector's network (no reference
 * counterpart: smf has no learned component). A one-hidden-layer MLP in
 * FP32, d features (<= 32) -> h ReLU units (<= 64) -> one logit, its
 * parameters packed as W1 (h x d, row-major), b1 (h), w2 (h), b2 (1):
 * smfg_mlp_params(d, h) floats. All pointers are device memory; the calls
 * are synchronous on the legacy default stream. forward: out[s] =
 * sigmoid(logit(X[s, :])). backward: grad (params + 1 floats, the last
 * the loss) of sum_s w_s BCE(p_s, y_s) / n (w NULL: 1), scratch holding
 * ceil(n / 128) * (params + 1) floats; the sum is taken in a fixed order.
 * adam: one Adam step (step >= 1 for the bias corrections). */
SMFG_API int smfg_mlp_params(int d, int h);
SMFG_API int smfg_mlp_forward(const float *d_X, int n, int d, const float *d_params, int h, float *d_out);
SMFG_API int smfg_mlp_backward(const float *d_X, const float *d_y, const float *d_w, int n, int d,
                               const float *d_params, int h, float *d_scratch, float *d_grad);
SMFG_API int smfg_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, int np, float lr,
                           float beta1, float beta2, float eps, int step);

/* A symbolic analysis of the engine's own (host code, no GPU needed),
 * producing the smfg_analysis_t contract above when smf's analyse
 * (solver/src/symbolic_analysis.cpp:434, out of this library's scope) is not
 * at hand: nested-dissection ordering, elimination tree, supernodes and
 * relaxed amalgamation. Input: lower CSC (0-based; entries above the
 * diagonal are mirrored, duplicates allowed). ordering: SMFG_ORDER_*. */
#define SMFG_ORDER_ND 0
#define SMFG_ORDER_NATURAL 1
#define SMFG_ORDER_ND_FINE 2
typedef struct smfg_symbolic_s *smfg_symbolic_t;
SMFG_API int smfg_analyse(int n, const int *col_ptr, const int *row_idx, int ordering, int nemin,
                          smfg_symbolic_t *out);
/* The same analysis on a caller-given fill-reducing ordering (perm[new] =
 * old, e.g. the permutation of smf's METIS analysis, AnalysisKeep::perm):
 * elimination tree, supernodes, amalgamation and front rows are built on it.
 * SMFG_ERR_INVALID_ARG when perm is not a permutation of 0..n-1. */
SMFG_API int smfg_analyse_ordered(int n, const int *col_ptr, const int *row_idx, const int *perm,
                                  int nemin, smfg_symbolic_t *out);
/* Pointers into the analysis (valid until smfg_symbolic_free); flops: the
 * delay-free factorization flops in smf's count; factor_entries: |L|. */
SMFG_API int smfg_symbolic_view(smfg_symbolic_t s, smfg_analysis_t *a, double *flops,
                                int64_t *factor_entries);
SMFG_API void smfg_symbolic_free(smfg_symbolic_t *s);

/* Tensor-core symmetric rank-k update with split products: the lower
 * triangle of the n x n matrix C minus L W^T (C, L, W in device memory,
 * column-major; L and W n x k). Each FP64 operand is split as hi + lo in
 * TF32 (SMFG_TC_TF32X3) or BF16 (SMFG_TC_BF16X3) and hi*hi + hi*lo + lo*hi
 * accumulate in FP32 on the tensor cores; the sum is subtracted from C in
 * FP64. The kernel of the mixed-precision path's trailing updates, exposed
 * for callers and tests. No reference counterpart: smf computes this
 * product in FP64 (schur_update, solver/src/ldlt_kernel.cpp:764-933).
 * Synchronous on the legacy default stream of the current device. */
#define SMFG_TC_TF32X3 0
#define SMFG_TC_BF16X3 1
SMFG_API int smfg_tc_update(double *d_C, int ldc, int n, const double *d_L, int ldl, const double *d_W,
                            int ldw, int k, int kind);
SMFG_API const char *smfg_error_string(int code);
/* Message of the last CUDA or internal error on the calling thread. */
SMFG_API const char *smfg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SMFG_H */
