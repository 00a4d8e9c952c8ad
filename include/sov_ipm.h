/*
 * sov_ipm.h -- C ABI of the B200 Mehrotra predictor-corrector interior-point engine.
 *
 * Plain C types only (fixed-width integers, doubles, raw pointers), so any host language that
 * can call C can bind it. Every entry point returns 0 on success or a negative SOV_E* code on an
 * argument / device error; the solve status itself is reported in sov_result.status.
 *
 * Reference interfaces replaced (paths inside the Abhishekmishra2808/sovereign tree):
 *   sov_lp_solve        <- sovereign::InteriorPointSolver::solve
 *                          solver/lp/include/sovereign/interior_point.hpp:26-36,
 *                          solver/lp/src/interior_point.cpp:747-757 (reached from
 *                          LpSolver::solve, solver/lp/src/lp_solver.cpp:59-62,70-72)
 *   sov_qp_solve        <- sovereign::QpInteriorPointSolver::solve
 *                          solver/qp/include/sovereign/qp_interior_point.hpp:21-31,
 *                          solver/qp/src/qp_interior_point.cpp:3123-3186 (generic path)
 *   sov_lp_solve_batch  <- no batched entry in the reference; replaces N independent
 *                          InteriorPointSolver::solve calls (e.g. MILP node LPs,
 *                          solver/milp/src/branch_and_bound.cpp:497)
 *   sov_device_info     <- sovereign::cuda::device_info / gpu_available
 *                          solver/gpu/include/sovereign/cuda_driver.hpp:14-40,
 *                          solver/gpu/include/sovereign/gpu_spmv.hpp:16-49
 *   sov_spmv_csc        <- sovereign::spmv_csc_auto (solver/gpu/src/gpu_spmv.cpp:70-102)
 *   sov_normal_factor_solve <- NormalEquations::factor + ::solve
 *                          (solver/lp/src/interior_point.cpp:163-182)
 *
 * Models cross the boundary in index form: variable j and row i of a sovereign::OptimizationModel
 * (solver/core/include/sovereign/types.hpp:53-59) become column j and row i here; the adapter in
 * sov_ipm_adapter.hpp maps names to indices and results back to name-keyed maps.
 */
#ifndef SOV_IPM_H
#define SOV_IPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* sovereign::SolverStatus, same order (types.hpp:20-30). */
enum {
  SOV_OPTIMAL = 0,
  SOV_FEASIBLE = 1,
  SOV_INFEASIBLE = 2,
  SOV_UNBOUNDED = 3,
  SOV_TIME_LIMIT = 4,
  SOV_ITERATION_LIMIT = 5,
  SOV_NUMERICAL_ERROR = 6,
  SOV_ERROR = 7,
  SOV_NOT_IMPLEMENTED = 8
};

/* sovereign::ConstraintSense (types.hpp:12). */
enum { SOV_LE = 0, SOV_GE = 1, SOV_EQ = 2 };

/* Return codes of the entry points (the solve outcome is in sov_result.status). */
enum {
  SOV_OK = 0,
  SOV_E_ARGUMENT = -1,   /* null pointer, negative size, inconsistent CSC */
  SOV_E_NO_DEVICE = -2,  /* no CUDA device or the sm_100a kernels cannot load */
  SOV_E_CUDA = -3,       /* a CUDA call failed; the message names it */
  SOV_E_TOO_LARGE = -4,  /* model exceeds the engine's size limits */
  SOV_E_UNSUPPORTED = -5, /* model shape this engine does not solve (message says why) */
  SOV_E_NUMERICAL = -6    /* a factorization met a non-finite pivot (NaN or Inf in the inputs) */
};

/* Arithmetic of the Newton solves. */
enum {
  SOV_PRECISION_FP64 = 0,  /* FP64 normal matrix, FP64 Cholesky, FP64 solves */
  SOV_PRECISION_MIXED = 1  /* FP32 normal matrix + FP32 (3xTF32 tensor-core) Cholesky as the
                              preconditioner of FP64 PCG; FP64 residuals, mu, sigma, ratio test */
};

/* Normal-equation factorization (the reference's SOVEREIGN_IPM_NORMAL_EQUATIONS knob). */
enum {
  SOV_FACTOR_AUTO = 0,   /* banded when the bandwidth is small, else dense */
  SOV_FACTOR_DENSE = 1,  /* dense m x m Cholesky (dense-Schur) */
  SOV_FACTOR_BANDED = 2, /* banded LDL^T in the natural row order */
  SOV_FACTOR_XSPACE = 3, /* QP only: eliminate the slacks and factor Q + H + A'ZW^-1A over the structural
                            columns (rows must all be inequalities, Q_jj > 0); exact Newton step, but
                            with FP64 iterates it stalls once slack weights exceed ~1e12 */
  SOV_FACTOR_SPARSE = 4  /* sparse L D L' on the GPU after a minimum-degree order (NormalEquations'
                            sparse path, interior_point.cpp:129-182, sparse_ldlt.cpp:19-223); AUTO takes
                            it when the normal matrix is too large for the dense factorization */
};

/* One LP or convex QP in index form.
 *   min/max  obj'x + 1/2 x'Qx + obj_constant
 *   s.t.     sum_j A[i][j] x_j  (<=, >=, =)  rhs[i]      (sense[i])
 *            lb[j] <= x_j <= ub[j]
 * A is column-compressed (CSC), m x n; duplicate (row, col) entries are summed.
 * lb <= -1e29 means no lower bound (QP only; the LP path shifts every column by lb);
 * ub >= 1e29 means no upper bound (interior_point.cpp:239, qp_interior_point.cpp:135-138).
 * Q (QP only, else NULL) holds the stored quadratic terms q_ij of Objective::quadratic
 * (types.hpp:43) column-compressed, each stored term once: the objective term is
 * 1/2 * sum over stored terms of q_ij x_i x_j (qp_interior_point.cpp:65-67). */
typedef struct sov_model {
  int32_t n;
  int32_t m;
  int32_t maximize;
  int32_t reserved;
  const int32_t* col_ptr;  /* n + 1 */
  const int32_t* row_idx;  /* nnz */
  const double* values;    /* nnz */
  const double* obj;       /* n */
  double obj_constant;
  const double* lb;        /* n */
  const double* ub;        /* n */
  const int8_t* sense;     /* m: SOV_LE / SOV_GE / SOV_EQ */
  const double* rhs;       /* m */
  const int32_t* q_col_ptr; /* n + 1, or NULL */
  const int32_t* q_row_idx;
  const double* q_values;
} sov_model;

/* Solver options; sov_default_lp_options / sov_default_qp_options give the reference defaults
 * (InteriorPointOptions, interior_point.hpp:7-24; QpInteriorPointOptions,
 * qp_interior_point.hpp:7-18). */
typedef struct sov_options {
  int32_t max_iterations;
  int32_t enable_scaling;
  double feasibility_tol;
  double optimality_tol;
  double fraction_to_boundary;
  int32_t precision;      /* SOV_PRECISION_* */
  int32_t factorization;  /* SOV_FACTOR_* */
  /* Optional warm start in the engine's internal standard form (scaled, shifted, slack columns
   * appended; sizes from sov_ipm_dims). NULL = Mehrotra-style start (interior_point.cpp:488-506).
   * A warm start that is worse than the default start is discarded. */
  const double* warm_x;   /* n_ipm */
  const double* warm_y;   /* m_ipm */
  const double* warm_s;   /* n_ipm */
  /* Mixed precision: cap on FP64 PCG iterations per Newton solve before the engine refactors in
   * FP64 for that iteration. */
  int32_t pcg_max_iterations;
  /* 0: sov_result.ipm_x/y/s receive the final iterate; k >= 1: the iterate at the start of
   * iteration k (k = 1 is the starting point), or the final one if the solve ends earlier. A point
   * on the central path's early stretch is the training target of the learned warm start. */
  int32_t ipm_iterate_at;
} sov_options;

/* Per-solve diagnostics (the fields of sovereign::LpDiagnostics, types.hpp:64-89, that the IPM
 * fills at interior_point.cpp:366-407,616-631,700-707). Optional: pass NULL to skip. */
#define SOV_HISTORY_MAX 128
typedef struct sov_diagnostics {
  int32_t scaling_applied;
  int32_t history_len;
  int32_t step_history_len;
  int32_t refactorizations;
  double coefficient_min_abs_before, coefficient_max_abs_before;
  double coefficient_min_abs_after, coefficient_max_abs_after;
  int64_t stall_iteration;
  double stall_gap, stall_mu, stall_primal_step, stall_dual_step;
  int64_t history_iterations[SOV_HISTORY_MAX];
  double objective_history[SOV_HISTORY_MAX];
  double gap_history[SOV_HISTORY_MAX];
  double mu_history[SOV_HISTORY_MAX];
  double primal_step_history[SOV_HISTORY_MAX];
  double dual_step_history[SOV_HISTORY_MAX];
  /* engine counters (no reference counterpart) */
  int32_t fp64_fallbacks;      /* mixed precision: iterations refactored in FP64 */
  int32_t pcg_iterations;      /* mixed precision: total PCG iterations */
  int32_t warm_start_used;     /* 1 when the supplied warm start was kept */
  int32_t structured_qp;       /* 1: the QP took the structured convex-sequence path; its dual map holds
                                  the model's rows only (qp_interior_point.cpp:2198-2202) */
} sov_diagnostics;

/* Result of one solve (sovereign::SolverResult, types.hpp:117-155, in index form).
 * primal / dual_col / dual_row / ipm_x / ipm_y / ipm_s are caller-allocated and may be NULL. */
typedef struct sov_result {
  int32_t status;              /* SOV_OPTIMAL ... */
  int32_t iterations;
  int32_t has_objective_value;
  int32_t n_ipm, m_ipm;        /* internal standard-form sizes */
  double objective_value;      /* on the original model, constant included */
  double duality_gap;          /* |x's| / (1 + |c'x|) on the scaled problem */
  double primal_residual;      /* ||b - Ax||_inf / max(1, ||b||_inf) */
  double dual_residual;        /* ||c - A'y - s||_inf / max(1, ||c||_inf) */
  double* primal;              /* n: x_j (= shift + col_scale * x_ipm) */
  double* dual_col;            /* n: dual slack s_j / col_scale_j, key = variable name */
  double* dual_row;            /* m: row_scale_i * y_i, key = "row_<i>" */
  double* ipm_x;               /* n_ipm: final internal iterate (training data for warm starts) */
  double* ipm_y;               /* m_ipm */
  double* ipm_s;               /* n_ipm */
  sov_diagnostics* diagnostics;
  double solve_seconds;        /* device time of the iteration loop */
  char message[512];
} sov_result;

void sov_default_lp_options(sov_options* opt);
void sov_default_qp_options(sov_options* opt);

/* Internal standard-form sizes of a model (LP: interior_point.cpp:250,312-314;
 * QP: qp_interior_point.cpp:155,195-197). */
int sov_ipm_dims(const sov_model* model, int32_t qp, int32_t* n_ipm, int32_t* m_ipm);

/* One LP through the GPU IPM. Synchronous; host pointers are borrowed for the call. */
int sov_lp_solve(const sov_model* model, const sov_options* opt, sov_result* result);

/* One convex QP through the GPU IPM (QpInteriorPointSolver::solve, qp_interior_point.cpp:3123-3186).
 * Separable (diagonal) Hessians take the y-space normal equations A (Q + X^-1 S)^-1 A'. A Hessian
 * that couples variables takes the quasi-definite KKT system [Q + X^-1 S + delta I, A'; A, -delta I]
 * as a sparse L D L' on the GPU (QpKkt, :415-655: signed pivots, delta escalation, refinement) when
 * Q is sparse, beyond 16384 IPM columns, or with SOV_FACTOR_SPARSE; small dense couplings are held
 * dense as H = Q + X^-1 S and reduced to A H^-1 A'. A free variable without curvature always takes
 * the KKT system. */
int sov_qp_solve(const sov_model* model, const sov_options* opt, sov_result* result);

/* count independent LPs in one persistent batched launch (one CTA per LP, the whole IPM loop
 * on the device). opt is one shared option block (opt_stride 0; NULL = LP defaults) or an array
 * of blocks opt_stride bytes apart, one per LP: per-LP tolerances, iteration limits, scaling and
 * warm starts (warm_x / warm_y / warm_s in the engine's standard form, taken under the same
 * safeguard as sov_lp_solve; diagnostics->warm_start_used reports it). LPs whose normal matrix
 * does not fit the batched kernel are solved one by one through sov_lp_solve. */
int sov_lp_solve_batch(int32_t count, const sov_model* models, const sov_options* opt,
                       int32_t opt_stride, sov_result* results);

/* A parametric family: count LPs that share the constraint matrix, bounds, row senses and sense
 * of optimisation (only obj, obj_constant and rhs differ), solved together -- one symbolic analysis
 * of the normal matrix for the family, and every kernel of an iteration (residuals, assembly of
 * A D_k A', the sparse L D L' and its solves, directions, ratio tests, update) running over up to 64
 * LPs at once with their vectors interleaved. Each LP follows sov_lp_solve's iteration, stopping
 * test, best-iterate rule and warm-start safeguard; opt / opt_stride as in sov_lp_solve_batch (the
 * LPs must agree on enable_scaling and fraction_to_boundary; precision and factorization are not
 * used: the path is FP64 sparse L D L'). solve_seconds of each result is its chunk's time. LPs
 * without rows go through sov_lp_solve. SOV_E_ARGUMENT when the models do not share the structure. */
int sov_lp_solve_family(int32_t count, const sov_model* models, const sov_options* opt, int32_t opt_stride,
                        sov_result* results);

/* Device-resident batch: prepare once (host standard form + upload), solve many times (device
 * only, stream-ordered), read back. Used to time the solver with inputs already in HBM. opt and
 * opt_stride as in sov_lp_solve_batch (one shared block, or one block per LP). */
typedef struct sov_batch sov_batch;
int sov_batch_create(int32_t count, const sov_model* models, const sov_options* opt,
                     int32_t opt_stride, sov_batch** out);
int sov_batch_solve(sov_batch* batch, void* cuda_stream);
int sov_batch_results(sov_batch* batch, sov_result* results);
/* Kernel launches issued by the last sov_batch_solve, and the device time of its kernels. */
int sov_batch_stats(const sov_batch* batch, int32_t* launches, double* kernel_ms,
                    double* algorithmic_bytes, double* algorithmic_flops);
/* Bytes the last sov_batch_create copied host->device and the last sov_batch_results copied
 * device->host (the end-to-end transfer volume of one batch). */
int sov_batch_transfer_bytes(const sov_batch* batch, double* h2d_bytes, double* d2h_bytes);
void sov_batch_destroy(sov_batch* batch);

/* Batched-kernel schedule chosen by the autotuner for a size bucket (threads per CTA, normal
 * matrix precision). tuning_file may be NULL (in-memory only). */
int sov_autotune(int32_t count, const sov_model* models, const sov_options* opt,
                 const char* tuning_file, char* report, int32_t report_len);

/* y = A x (transpose = 0) or y = A' x (transpose = 1) for a CSC matrix, FP64, on the GPU.
 * Host buffers in and out. Mirrors spmv_csc_auto (gpu_spmv.cpp:70-102). */
int sov_spmv_csc(int32_t nrows, int32_t ncols, const int32_t* col_ptr, const int32_t* row_idx,
                 const double* values, const double* x, double* y, int32_t transpose);

/* Factor M = A diag(d) A' + 1e-12 I (interior_point.cpp:74-101,163-180) on the GPU and solve
 * M z = rhs for nrhs right-hand sides (column-major m x nrhs, overwritten by z). Dependent rows
 * are dropped as the reference's tiny-pivot rule does (sparse_ldlt.cpp:165-173). */
int sov_normal_factor_solve(int32_t m, int32_t n, const int32_t* col_ptr, const int32_t* row_idx,
                            const double* values, const double* d, int32_t precision,
                            int32_t factorization, double* rhs, int32_t nrhs,
                            int32_t* dropped_pivots);

/* No counterpart in the reference. For callers that cannot let the library allocate device
 * memory (applications that own all device memory through their own pool, or run close to the
 * memory limit): the dense FP64 factor of A diag(d) A' + 1e-12 I and the solve for nrhs
 * right-hand sides, like sov_normal_factor_solve, but col_ptr, row_idx, values, d and rhs
 * (column-major m x nrhs, overwritten by the solution) are DEVICE pointers, rows within a column
 * must be distinct, and the work runs on cuda_stream. The device arrays cannot be checked on the
 * host: entries whose row lies outside [0, m), and columns whose col_ptr decreases, are skipped on
 * the device and the call returns SOV_E_ARGUMENT; col_ptr[n] must not exceed the length of
 * row_idx and values. A non-finite pivot returns SOV_E_NUMERICAL. The normal matrix is summed
 * with FP64 atomics, so results can differ from run to run in the last bits (the allocating
 * entry point sums in a fixed order). It calls no cudaMalloc or cudaFree: its
 * working storage is one fixed device array sized for m <= SOV_NOALLOC_MAX_ROWS (about 2.3 MB,
 * held by every GPU that loads the library until the process exits); larger m returns
 * SOV_E_TOO_LARGE. The first call on a device looks that array up (cudaGetSymbolAddress), so it
 * should come before any stream capture on that device. Calls share the array: two calls whose
 * work overlaps on the GPU race and must be ordered by the caller. The call returns after the
 * stream has finished this work; dropped_pivots is a host pointer (or NULL). */
#define SOV_NOALLOC_MAX_ROWS 512
int sov_normal_factor_solve_noalloc(int32_t m, int32_t n, const int32_t* col_ptr, const int32_t* row_idx,
                                    const double* values, const double* d, double* rhs, int32_t nrhs,
                                    int32_t* dropped_pivots, void* cuda_stream);

/* Warm-start network (no counterpart in the reference): an MLP n_in -> hidden x hidden_layers
 * (ReLU) -> n_out with FP32 master weights and BF16 tensor-core products (FP32 accumulate),
 * trained with Adam on mean-squared error. Parameters are laid out layer by layer as W (out x in,
 * row-major) then b. Host buffers in and out; row-major batches. */
typedef struct sov_mlp sov_mlp;
int sov_mlp_create(int32_t n_in, int32_t hidden, int32_t hidden_layers, int32_t n_out, uint64_t seed,
                   sov_mlp** out);
int64_t sov_mlp_param_count(const sov_mlp* mlp);
int sov_mlp_get_params(const sov_mlp* mlp, float* params, int64_t count);
int sov_mlp_set_params(sov_mlp* mlp, const float* params, int64_t count);
int sov_mlp_forward(sov_mlp* mlp, const float* x, int32_t batch, float* y);
/* Warm starts for a batch in one call, normalization and decoding on the GPU: the network input is
 * (params - in_mean) / in_std (FP64, rounded to FP32); its output o, with 2 n_ipm + m_ipm columns
 * (log x, y, log s normalized), becomes v = o * out_std + out_mean, and x = max(exp(clip(v, -40,
 * 40)), delta), y = v, s likewise, into x (batch x n_ipm), y (batch x m_ipm), s (batch x n_ipm),
 * row-major host arrays. */
int sov_mlp_predict_start(sov_mlp* mlp, const double* params, int32_t batch, const double* in_mean,
                          const double* in_std, const double* out_mean, const double* out_std, int32_t n_ipm,
                          int32_t m_ipm, double delta, double* x, double* y, double* s);
/* sov_lp_solve_batch with every LP started from the network's prediction for its parameters (row k
 * of params, batch = count), without the starts leaving the device: the prediction as in
 * sov_mlp_predict_start, then each LP's start gathered into the batch on the GPU. One options block
 * (or NULL) for all LPs; its warm_x/y/s are ignored. Every LP's IPM form must have n_ipm columns
 * and m_ipm rows (else SOV_E_ARGUMENT); each start is judged by the batch's safeguard like a
 * caller's. LPs the batched kernel does not take (more than 128 IPM rows) get their start copied
 * to the host and passed to the single-problem engine as its warm start. Results are those of
 * sov_lp_solve_batch given the same starts from host arrays. */
int sov_lp_solve_batch_predicted(sov_mlp* mlp, const double* params, const double* in_mean, const double* in_std,
                                 const double* out_mean, const double* out_std, int32_t n_ipm, int32_t m_ipm,
                                 double delta, int32_t count, const sov_model* models, const sov_options* opt,
                                 sov_result* results);
/* loss = mean((f(x) - t)^2); grad (param_count floats, or NULL) = its gradient */
int sov_mlp_loss_grad(sov_mlp* mlp, const float* x, const float* t, int32_t batch, double* loss, float* grad);
/* epochs of shuffled mini-batches over count samples; final_loss = mean loss of the last epoch */
int sov_mlp_train(sov_mlp* mlp, const float* x, const float* t, int32_t count, int32_t epochs, int32_t batch,
                  float lr, uint64_t seed, double* final_loss);
void sov_mlp_destroy(sov_mlp* mlp);

/* Certificate of an answer against the original model, computed on the GPU (verify.cu): the
 * checks of sovereign::SolutionVerifier::verify (solver/core/src/verifier.cpp:10-150; default
 * tolerance 1e-6 there) and the dual side an interior point carries, so that an IPM answer can be
 * accepted without a simplex crossover. result must hold primal (n) and dual_row (m: the published
 * "row_<i>" multipliers of the minimisation form), status, objective_value and duality_gap. */
enum {
  SOV_CERT_NO_FEASIBLE_STATUS = 1, /* status gives no feasible primal (verifier.cpp:17-27) */
  SOV_CERT_UNCHECKABLE_STATUS = 2, /* INFEASIBLE / UNBOUNDED without a certificate (:29-38) */
  SOV_CERT_NONFINITE = 4,          /* a non-finite primal value or row activity */
  SOV_CERT_BOUND = 8,              /* max bound violation > tol */
  SOV_CERT_CONSTRAINT = 16,        /* max row violation > tol */
  SOV_CERT_OBJECTIVE = 32,         /* reported objective differs from the recomputed one by > tol (1 + |obj|) */
  SOV_CERT_GAP = 64                /* OPTIMAL with a reported duality gap > tol */
};
typedef struct sov_certificate {
  int32_t is_valid;                 /* the verifier's verdict: no issue bit set */
  int32_t issues;                   /* SOV_CERT_* bits */
  int32_t nonfinite;                /* non-finite primal values and row activities */
  int32_t reserved;
  double max_bound_violation;       /* max(0, max_j max(lb_j - x_j, x_j - ub_j)) */
  double max_constraint_violation;  /* max(0, max_i (<=: a_i x - b_i, >=: b_i - a_i x, =: |a_i x - b_i|)) */
  double recomputed_objective;      /* constant + c'x + 1/2 sum of stored q_ij x_i x_j */
  double dual_objective;            /* b'y - 1/2 x'Qx + sum_j (lb_j max(d_j, 0) + ub_j min(d_j, 0)), model sense */
  double max_dual_infeasibility;    /* sign violations of d = c + Qx - A'y (min form) and of y */
  double relative_gap;              /* |primal - dual objective| / (1 + |primal|) */
} sov_certificate;
int sov_verify_solution(const sov_model* model, const sov_result* result, double tol, sov_certificate* cert);

/* Model ingest without name-keyed maps: the reference's JSON model format
 * (solver/core/src/json_io.cpp:13-80, load_model_from_json_file / _string, :112-130) parsed in one
 * pass straight into the index form above (A column-compressed, rows ascending in each column).
 * Unknown variables in a constraint return SOV_E_ARGUMENT with the IPM's message ("Unknown
 * variable in constraint: <name>"); parse errors name the byte offset. The handle owns the arrays;
 * sov_json_model_view stays valid until sov_json_model_destroy. Host only (no GPU needed). */
typedef struct sov_json_model sov_json_model;
int sov_model_from_json(const char* text, size_t len, sov_json_model** out);
const sov_model* sov_json_model_view(const sov_json_model* jm);
int32_t sov_json_model_problem_type(const sov_json_model* jm);          /* 0 LP, 1 QP, 2 MILP */
int32_t sov_json_model_variable_type(const sov_json_model* jm, int32_t j); /* 0 continuous, 1 integer, 2 binary */
const char* sov_json_model_variable_name(const sov_json_model* jm, int32_t j);
const char* sov_json_model_row_name(const sov_json_model* jm, int32_t i);
void sov_json_model_destroy(sov_json_model* jm);

/* LP presolve and postsolve in index form (presolve.cpp; the reference presolves every LP in its
 * engine, solver/core/src/engine.cpp:108-176, with solver/presolve/src/presolve.cpp): fixed columns,
 * empty rows, singleton rows (to bounds) and empty columns, repeated until nothing changes.
 * sov_presolve_lp borrows `model` for the handle's lifetime; sov_presolve_reduced is the model to
 * solve (when the info status is -1; otherwise presolve decided: OPTIMAL with every column fixed,
 * INFEASIBLE or UNBOUNDED); sov_postsolve_lp maps a reduced result (or none, when presolve
 * decided) back to the original columns and rows: primal, row multipliers (removed singleton rows
 * recover theirs from their column's reduced cost), reduced costs, and the objective evaluated on
 * the original model. Host only. sov_lp_solve_presolved does all three around sov_lp_solve and,
 * as the reference's engine does (engine.cpp:160-176), solves the original model again when
 * presolve claims infeasibility or its answer violates the original rows by more than 1e-6
 * relative (the message then says so). */
typedef struct sov_presolve sov_presolve;
int sov_presolve_lp(const sov_model* model, sov_presolve** out);
const sov_model* sov_presolve_reduced(const sov_presolve* pre);
int sov_presolve_info(const sov_presolve* pre, int32_t* status, int32_t* rows_removed, int32_t* cols_removed,
                      int32_t* bounds_tightened, char* message, int32_t message_len);
int sov_postsolve_lp(const sov_presolve* pre, const sov_result* reduced, sov_result* full);
void sov_presolve_destroy(sov_presolve* pre);
int sov_lp_solve_presolved(const sov_model* model, const sov_options* opt, sov_result* result);

/* Device name, SM count, memory; returns SOV_E_NO_DEVICE when no usable sm_100 GPU exists. */
int sov_device_info(char* buf, int32_t len);

/* Last error message of this thread. */
const char* sov_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SOV_IPM_H */
