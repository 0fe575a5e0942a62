/*
 * xplus_b200.h -- C ABI of the B200 Jacobi-PCG solver.
 *
 * A drop-in for the PCG path of project-xplus: caller-owned host arrays in, the
 * library owns device memory, one CUDA stream per handle, no CPU fallback (every
 * compute entry point fails with XPLUS_ERR_CUDA when no usable sm_100 device is
 * present).  Not thread-safe per handle.  All entry points return an int status
 * (XPLUS_OK or an XPLUS_ERR_* code) unless stated otherwise; the text of the last
 * error on the calling thread is returned by xplus_last_error_string().
 *
 * Reference interfaces replaced (paths are within the reference project):
 *   solver entry   SolverConfig{tau,max_iters}      include/cg_common.hpp:52-55
 *                  run_defaults::kTau/kMaxIters      host/run_defaults.hpp:12-13
 *                  CuperPcgResult / GoldenResult     host/cuper_pcg_solver.hpp:62-73,
 *                                                    src/CgSolverGolden.hpp:24-31
 *   single launch  cuper_pcg_control_kernel(...)     kernels/cuper_pcg_control_kernel.cpp:972-1001
 *                  status[0..1], metrics[0..3]       kernels/cuper_pcg_control_kernel.cpp:1229-1234
 *   multi-kernel   spmv_csr_kernel ... update_p_kernel  archived/include/cg_kernels.hpp:9-54
 *   loader         CsrDataset::load                  src/CsrDataset.hpp:19-67
 *   jacobi         extract_jacobi_diag / build_jacobi_inverse
 *                                                    src/CsrDataset.hpp:92-116, host/pcg_common.hpp:42-54
 *   packed format  build_cuper_control_matrix        host/cuper_control_matrix.hpp:130-207
 */
#ifndef XPLUS_B200_H
#define XPLUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status of a solve: same codes as kernels/cuper_pcg_control_kernel.cpp:90-94,
 *      plus XPLUS_TIMEOUT for a grid barrier that gave up waiting ---- */
#define XPLUS_CONVERGED 0
#define XPLUS_MAX_ITER 1
#define XPLUS_BREAKDOWN 2
#define XPLUS_TIMEOUT 3

/* ---- return codes of API calls ---- */
#define XPLUS_OK 0
#define XPLUS_ERR_ARG 10     /* invalid argument (null pointer, n <= 0, tau <= 0, ...) */
#define XPLUS_ERR_CUDA 11    /* CUDA runtime error or no usable device */
#define XPLUS_ERR_DATA 12    /* invalid CSR, missing or zero diagonal (the loader's throws) */
#define XPLUS_ERR_IO 13      /* file could not be opened / parsed */
#define XPLUS_ERR_NOMEM 14   /* host or device allocation failed */

/* ---- element types ---- */
#define XPLUS_F32 0
#define XPLUS_BF16 1
#define XPLUS_F64 2
#define XPLUS_F16 3          /* FP16 values with one power-of-two scale per matrix (row-sum form) */

/* ---- tolerance semantics ---- */
#define XPLUS_TAU_ABS_RR 0   /* stop when the recurrence rr = ||r||^2 <= tau (the reference's
                                test, src/CgSolverGolden.hpp:74-76,112) */
#define XPLUS_TAU_REL_TRUE 1 /* stop when the FP64 true residual ||b - A x|| / ||b|| <= tau,
                                using FP64 residual replacement (requires the FP64 matrix copy) */

/* ---- preconditioners ---- */
#define XPLUS_PREC_JACOBI 0
#define XPLUS_PREC_GTG 1     /* M^-1 = G^T G, G lower-triangular on A's lower pattern */

typedef struct xplus_opts {
    int value_type;        /* XPLUS_F32 | XPLUS_BF16 | XPLUS_F16 | XPLUS_F64: matrix values in the
                              SpMV.  The 16-bit types need row_sum_form.  FP16 (11-bit significand,
                              values divided by one power-of-two scale) keeps stiffness matrices
                              within ~1% of A; BF16 (8-bit) perturbs them by ~4%, which stalls or
                              diverges the inner PCG on large FEM systems */
    int vector_type;       /* XPLUS_F32 | XPLUS_F64: x, r, p, Ap storage in the inner loop */
    int slice_height;      /* SELL-C-sigma C; must be 32 */
    int sigma;             /* SELL sort window (rows); multiple of 32, or 1 for no sorting */
    int chunk;             /* entries per row per vector load: 1, 2 or 4 (default 4) */
    int keep_fp64;         /* keep an FP64 copy of A for true residuals (forced on for TAU_REL_TRUE) */
    int replace_every;     /* FP64 residual replacement every k iterations (0: only on stagnation
                              / at convergence) */
    double replace_drop;   /* also replace when ||r|| fell by this factor since the last
                              replacement (default 1e-2); 0 disables.  With FP32 vectors the
                              recurrence residual stalls near 1e-7 of its start, so TAU_REL_TRUE
                              solves need a replacement before that point */
    int block_threads;     /* threads per CTA of the persistent kernel (0: auto) */
    int blocks_per_sm;     /* CTAs per SM (0: occupancy-derived) */
    double barrier_timeout_s; /* a grid barrier gives up after this long: status XPLUS_TIMEOUT */
    int device;            /* CUDA device ordinal */
    int row_sum_form;      /* FP32/BF16 values: store off-diagonal weights w_ij and row sums
                              s_i = sum_j a_ij, and compute y_i = s_i x_i + sum_j w_ij (x_j - x_i)
                              (default 1).  Rounding then perturbs each weight and each row sum
                              relatively, so the stored operator stays spectrally close to A;
                              rounding a_ii instead shifts the near-null space of a stiffness
                              matrix and multiplies the iteration count */
    int index16;           /* store columns as int16 offsets from the row when every |col - row|
                              < 32768 after ordering (lossless; default 1) */
    int l2_persist;        /* mark the matrix stream as persisting in L2 for the solve launch
                              (default 1).  Raises this process's persisting-L2 limit while the
                              handle exists; destroying the handle releases its persisting lines
                              and the last such handle restores the previous limit */
    int resident;          /* FP32 vectors, row-sum form: use the SM-resident kernel (state and
                              the search direction's band + halo in shared memory) when one CTA
                              per SM holds it (default 1) */
    int restart_on_replace; /* search direction after an FP64 residual replacement: 0 keeps it,
                              1 restarts it (p = z) after every replacement, 2 restarts it only
                              after replacements triggered by a replace_drop fall of ||r|| or by
                              the convergence check (periodic ones, replace_every, keep it),
                              3 adaptive: starts as 2 and switches to 1 for the rest of the solve
                              when ||b - A x|| grows past twice its best or stagnation_window
                              replacements bring no progress, 4 flexible: at every replacement
                              p is re-conjugated to the replaced residual with the flexible-CG
                              coefficient beta = -(z.Ap)/(p.Ap), switching to 1 for the rest of
                              the solve on the same two signals as 3.
                              -1 (default): 4 for 16-bit values, whose inexact operator opens a
                              gap between the recurrence and the true residual that a kept p
                              does not survive, 0 otherwise */
    int barriers_per_iter; /* SM-resident kernel: 1 (default) folds both dot products into one
                              reduction by expanding r_{k+1}.z_{k+1} and r_{k+1}.r_{k+1} in alpha;
                              2 reduces them after the update as the reference does */
    double stagnation_gain; /* TAU_REL_TRUE: an FP64 replacement counts as progress when it lowers
                              the best ||b - A x|| by this fraction (default 0.05) ... */
    int stagnation_window; /* ... and this many replacements in a row without progress stop the
                              solve (status XPLUS_MAX_ITER, metrics.reserved[0] = 1; default 8) */
    int build_on_gpu;      /* xplus_pcg_create builds the SELL-C-sigma layout on the GPU (the
                              same arrays as the host builder, bit for bit; default 1, sigma <=
                              4096); 0 builds it on the host */
    double split_ratio;    /* 16-bit values, xplus_pcg_create: an off-diagonal entry a_ij of a
                              row i or j whose sum_k |a_ik| / a_ii exceeds this, with |a_ij|
                              above half of min(a_ii, a_jj), is stored as two 16-bit terms, the
                              rounded value and its rounding remainder, in two slots of the row
                              (the FP64 copy holds both terms, summing to a_ij exactly).  Such
                              rows carry large weights of both signs that cancel in A but whose
                              16-bit rounding errors do not; left rounded they can make the
                              stored operator indefinite.  0: off; -1 (default): 1.5 for BF16,
                              2 for FP16 values.  Measured on the 128^3 P1-tetrahedra system
                              (1e-10, replacement every 50 iterations or at a 1e-4 drop): BF16
                              826 iterations in 102 ms with 1.6% more slots (singly rounded BF16
                              diverges), FP16 836 in 91 ms, FP32 values 807 in 90 ms */
} xplus_opts;

typedef struct xplus_metrics {
    int status;            /* XPLUS_CONVERGED .. XPLUS_TIMEOUT */
    int iterations;        /* inner PCG iterations (status[1] of the control kernel) */
    int replacements;      /* FP64 residual replacements performed */
    int reserved0;
    double rz, rr, pap, alpha;  /* metrics[0..3] of the control kernel */
    double true_rel_residual;   /* FP64 ||b - A x|| / ||b|| at exit (when the FP64 copy exists) */
    double kernel_ms;           /* device time of the solve launch(es) */
    double setup_ms;            /* host+device time of xplus_pcg_create */
    double reserved[4];         /* [0] stagnation stop (1/0), [1] device time from the kernel's
                                   own clock (ms), [2] kernel: 0 global-memory persistent,
                                   1 SM-resident two-barrier, 2 SM-resident one-barrier */
} xplus_metrics;

typedef struct xplus_pcg xplus_pcg;      /* one SPD system resident on one GPU */

void xplus_opts_default(xplus_opts* opts);
const char* xplus_last_error_string(void);
const char* xplus_version(void);
/* Number of sm_100 devices visible (0 when none); never fails. */
int xplus_device_count(void);

/* ------------------------------------------------------------------------------------
 * Single-system solver: replaces the XRT launch of cuper_pcg_control_kernel
 * (host/cuper_control_xrt_host.cpp:205-272) and the host loops of
 * run_local_multi_kernel_solver / run_cuper_pcg_solver.
 * ------------------------------------------------------------------------------------ */

/* Build SELL-C-sigma, Jacobi inverse and upload.  CSR as CsrDataset holds it
 * (row_ptr[n+1], col_idx[nnz], values[nnz], FP64).  Errors: XPLUS_ERR_DATA for the
 * loader/diagonal conditions of src/CsrDataset.hpp:25-64,92-116. */
int xplus_pcg_create(const int* row_ptr, const int* col_idx, const double* values, int n,
                     const xplus_opts* opts, xplus_pcg** out);
int xplus_pcg_destroy(xplus_pcg* h);

/* Blocking solve with host arrays.  x0 may be NULL (zeros).  max_iters <= 0 means
 * max(4n, 1000) as src/CgSolverGolden.hpp:47.  resid_hist (nullable, length hist_len)
 * receives sqrt(rr) after each iteration, the per-iteration residual of the golden
 * trace (src/CgSolverGolden.hpp:101-108).  metrics may be NULL. */
int xplus_pcg_solve(xplus_pcg* h, const double* b, const double* x0, double tau, int tau_mode,
                    int max_iters, double* x_out, int* iters_out, double* resid_hist,
                    int hist_len, xplus_metrics* metrics);

/* Asynchronous solve on device-resident FP64 b and x (original row order), enqueued on
 * `stream` (a cudaStream_t, NULL = the handle's stream) without waiting for the device: the
 * relative tolerance is scaled by ||b||^2 summed inside the kernel, so b may be produced by
 * earlier work on the same stream.  d_x holds x0 on entry and x on exit.  Fetch the outcome
 * with xplus_pcg_last_metrics() (which waits for the solve).  d_b and d_x must be device (or
 * managed) memory of the handle's GPU: host or other-GPU pointers return XPLUS_ERR_ARG before
 * anything is enqueued. */
int xplus_pcg_solve_device(xplus_pcg* h, const double* d_b, double* d_x, double tau,
                           int tau_mode, int max_iters, void* stream);
int xplus_pcg_last_metrics(xplus_pcg* h, xplus_metrics* metrics);
/* Phase clock of the last solve, read from block 0's %globaltimer (ms, summed over the
 * iterations): {phase A work, grid-barrier wait after A, phase B work, wait after B}; for the
 * one-barrier SM-resident kernel {publishing the dot-product partials, barrier wait and
 * totals, pending update + new search direction (the CTA's own rows from shared memory, the
 * halo from the records), A p' from shared memory with each row's records and dot-product
 * terms}; for the G^T G
 * kernel {A p', all grid-barrier waits, x/r update + t = G r', z = G^T t}. */
int xplus_pcg_last_phase_times(xplus_pcg* h, double* ms4);
/* The same phase clock for every CTA of the last solve: ms[4*b + k], k as above; *blocks is
 * the grid size (pass ms = NULL to query it). */
int xplus_pcg_last_block_times(xplus_pcg* h, double* ms, int max_blocks, int* blocks);
/* Per-iteration trace of the last xplus_pcg_solve that asked for a history: rows x 5
 * doubles {alpha, beta, rz, rr, sqrt(rr)}, the fields of GoldenIterationTrace
 * (src/CgSolverGolden.hpp:15-22).  rows <= the hist_len of that solve. */
int xplus_pcg_last_trace(xplus_pcg* h, double* trace, int rows);

/* Test-only fault injection: in the next solves, CTA `block` withholds its arrival at
 * the first grid barrier, so every wait runs into its barrier_timeout_s bound and the
 * solve ends with status XPLUS_TIMEOUT (the context stays usable).  -1 switches it off. */
int xplus_pcg_debug_skip_arrival(xplus_pcg* h, int block);

/* y = A x through the handle's SELL matrix, FP64 host vectors in original row order. */
int xplus_pcg_spmv(xplus_pcg* h, const double* x, double* y);
/* y = A x on device vectors in SELL (permuted) order, of the handle's vector type, n_pad long,
 * enqueued on `stream`.  For bandwidth measurement. */
int xplus_pcg_spmv_device(xplus_pcg* h, const void* d_x, void* d_y, void* stream);
/* Sizes of the resident system: n, n_pad (SELL rows), nnz, stored slots (incl. padding),
 * and the bytes one SpMV must move in the stored format, padding excluded: stored entries x
 * (value + index bytes) + n x (x read + y write [+ row sum in the row-sum form]). */
int xplus_pcg_info(xplus_pcg* h, int64_t* n, int64_t* n_pad, int64_t* nnz, int64_t* slots,
                   int64_t* spmv_bytes);
/* Device buffers of the SELL vectors (n_pad elements of the vector type), for tests and
 * benchmarks that drive xplus_pcg_spmv_device. */
int xplus_pcg_scratch_vectors(xplus_pcg* h, void** d_x, void** d_y);
/* Control-kernel ABI (kernels/cuper_pcg_control_kernel.cpp:972-1001) on device pointers:
 * b and x are FP64 device vectors of length n in original order (x holds x0 on entry);
 * metrics[4] = {rz, rr, pAp, alpha} and status[2] = {code, iterations} are device
 * arrays.  The matrix, its Jacobi inverse and the work vectors are the handle's: m_inv,
 * r, z, p and ap are accepted for signature compatibility and are not touched (the
 * reference uses them only as workspace).  Tolerance semantics are the reference's
 * (rr <= tau).  Invalid parameters give status {2, 0} and zeroed metrics, as the
 * reference does (:1078-1087). */
int xplus_pcg_control(xplus_pcg* h, const double* b, const double* m_inv, double* x, double* r,
                      double* z, double* p, double* ap, double* metrics, int* status,
                      double tau, int max_iters, int n, void* stream);

/* ------------------------------------------------------------------------------------
 * Factorized preconditioner M^-1 = G^T G (no counterpart in the reference, whose only
 * preconditioner is Jacobi, host/pcg_common.hpp:42-54).  G is lower-triangular on A's lower
 * pattern in the row order given to xplus_pcg_create; its values are passed in "g_low" order:
 * A's CSR order of the entries with col <= row (n_glow values, the diagonal included).  The
 * solve applies G^T G as two more sliced SpMVs (no triangular solves) and keeps the FP64
 * residual replacement; Jacobi-PCG takes over inside the same launch when the G^T G solve
 * stagnates or reaches fallback_iters iterations (0: only on stagnation).  Needs FP32 vectors,
 * FP32, BF16 or FP16 values, row_sum_form and keep_fp64.  reserved[3] of the metrics holds the
 * iteration of the switch to Jacobi (-1: none).
 * ------------------------------------------------------------------------------------ */
/* G from host values (g_low NULL: back to Jacobi).  row_ptr / col_idx: the CSR pattern given
 * to xplus_pcg_create (the G layouts are built from it once). */
int xplus_pcg_set_gtg(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* g_low,
                      int fallback_iters);
/* G predicted on the GPU by the learned network (parameters as xplus_gnn_get_params returns
 * them) from the CSR given to xplus_pcg_create, its rows then scaled on the GPU to
 * (G A G^T)_ii = 1 (the network fixes each row's direction; the scale is the normalization
 * FSAI carries by construction).  XPLUS_ERR_DATA when a row has (G A G^T)_ii <= 0.  infer_ms
 * (nullable) gets the host+device time of the inference. */
int xplus_pcg_set_gnn(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* values,
                      const float* params, int fallback_iters, double* infer_ms);
/* xplus_pcg_set_gnn (which is this with refine_sweeps = 4) with the number of refinement sweeps
 * (0..16) run on the GPU between inference and normalization: each sweep takes the lower
 * entries j of every row i in ascending order and sets Ghat_ij to the minimizer of the row's
 * quadratic form (G A G^T)_ii at fixed Ghat_ii, a Gauss-Seidel step on the row's FSAI system
 * A[P_i, P_i] g = e_i.  Every step lowers the row's Kaporin term, so a sweep never makes a row
 * worse; it fixes rows the network cannot resolve, chiefly the two ends of a very stiff
 * element (a_ij^2 close to a_ii a_jj), where the row's best ratio G_ij / G_ii is sharp.
 * Repeated sweeps approach the exact FSAI row; from the network's G four sweeps come within
 * 1% of FSAI's iteration count on the 1108x1108 system, where from Jacobi ten are needed. */
int xplus_pcg_set_gnn_ex(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* values,
                         const float* params, int fallback_iters, int refine_sweeps, double* infer_ms);
/* The handle's current G in g_low order (g_low NULL: only *n_glow). */
int xplus_pcg_get_gtg(xplus_pcg* h, double* g_low, int64_t* n_glow);
/* Rescales the rows of the handle's current G (learned or given) to (G A G^T)_ii = 1, the
 * normalization FSAI carries by construction, from the CSR given to xplus_pcg_create (host,
 * threaded; G is read back from and written to the device).  XPLUS_ERR_DATA when a row has
 * (G A G^T)_ii <= 0. */
int xplus_pcg_scale_gtg(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* values);
/* Exact factorized sparse approximate inverse on A's lower pattern (host, no GPU): row i
 * solves A[P_i, P_i] g = e_i over P_i = {j <= i : a_ij != 0}, scaled to (G A G^T)_ii = 1.
 * The non-learned G of the same form, in g_low order. */
int xplus_fsai_lower(int n, const int* row_ptr, const int* col_idx, const double* values, double* g_low);

/* ------------------------------------------------------------------------------------
 * Learned-preconditioner trainer (no counterpart in the reference).  A 3-layer message-
 * passing network (hidden width 32) over A's graph predicts G: inputs log a_ii (centred),
 * sum_j |a_ij| / a_ii - 1 and a_ij / sqrt(a_ii a_jj); separate message weights for lower
 * and upper neighbours; G_ij = (w . relu(P h_i + bp + Q h_j + c e_ij + c2 f_ij) + bw) / sqrt(a_jj)
 * with f_ij = sum_{m < i, m != j} e_jm e_mi (two-step paths from j to i through i's other
 * lower neighbours, e the scaled off-diagonal entries),
 * G_ii = exp(wd . h_i + bwd) / sqrt(a_ii).  Two losses (xplus_gnn_set_loss):
 *   XPLUS_GNN_LOSS_PROBE    sum_p ||G A G^T v_p - v_p||^2 / (K n) over K probe vectors
 *                           v ~ N(0, I) (the default of a new trainer);
 *   XPLUS_GNN_LOSS_KAPORIN  (1/n) sum_i [log (G A G^T)_ii - 2 log Ghat_ii], Ghat = G D^1/2:
 *                           per row log(g A g / g_ii^2) on the row's pattern, free of the
 *                           row's scale and smallest at the exact FSAI row; summed, n log of
 *                           Kaporin's condition number of G A G^T once rows are normalized.
 * Forward, backward and Adam run on the GPU (FP32 arithmetic, parameters rounded to BF16 in
 * the forward pass, FP32 master copy).
 * ------------------------------------------------------------------------------------ */
#define XPLUS_GNN_LOSS_PROBE 0
#define XPLUS_GNN_LOSS_KAPORIN 1
typedef struct xplus_gnn_trainer xplus_gnn_trainer;
/* Number of parameters (floats); returns the count, not a status. */
int xplus_gnn_param_count(void);
/* Training systems as CSR (like xplus_batch_create); `probes` = K per step (1..64). */
int xplus_gnn_trainer_create(int nsys, const int* const* row_ptrs, const int* const* col_idxs,
                             const double* const* values, const int* ns, int probes, int device,
                             xplus_gnn_trainer** out);
int xplus_gnn_trainer_destroy(xplus_gnn_trainer* t);
/* Parameters in and out (FP32 master copy); setting them resets the Adam state. */
int xplus_gnn_set_params(xplus_gnn_trainer* t, const float* params);
int xplus_gnn_get_params(xplus_gnn_trainer* t, float* params);
/* Loss on system `sys` with the probes of `seed`, and its gradient (grad nullable). */
int xplus_gnn_loss_grad(xplus_gnn_trainer* t, int sys, uint64_t seed, double* loss, float* grad);
/* Loss of the trainer's later xplus_gnn_loss_grad / xplus_gnn_train calls
 * (XPLUS_GNN_LOSS_PROBE or XPLUS_GNN_LOSS_KAPORIN; the Kaporin loss ignores seeds). */
int xplus_gnn_set_loss(xplus_gnn_trainer* t, int kind);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) with a caller-given gradient. */
int xplus_gnn_adam(xplus_gnn_trainer* t, const float* grad, double lr);
/* `steps` Adam steps, one system per step (a seeded shuffle every epoch), probes from `seed`
 * and the step, learning rate cosine-decayed from lr to lr_final; losses (nullable) gets the
 * loss of every step. */
int xplus_gnn_train(xplus_gnn_trainer* t, int steps, double lr, double lr_final, uint64_t seed, double* losses);
/* Steps [first_step, first_step + steps) of a cosine learning-rate schedule over total_steps
 * (xplus_gnn_train is the window [0, steps) of a schedule of `steps`): training in windows
 * over successive sets of resident systems (xplus_gnn_trainer_load) follows one schedule. */
int xplus_gnn_train_window(xplus_gnn_trainer* t, int steps, double lr, double lr_final, uint64_t seed,
                           int64_t first_step, int64_t total_steps, double* losses);
/* Replaces the resident training systems (same CSR arguments as xplus_gnn_trainer_create);
 * parameters, the Adam state and the loss kind are kept, the workspace grows as needed. */
int xplus_gnn_trainer_load(xplus_gnn_trainer* t, int nsys, const int* const* row_ptrs,
                           const int* const* col_idxs, const double* const* values, const int* ns);
/* G of system `sys` under the current parameters as the network outputs it (rows not
 * normalized), in g_low order (g_low NULL: only *n_glow). */
int xplus_gnn_predict(xplus_gnn_trainer* t, int sys, double* g_low, int64_t* n_glow);

/* ------------------------------------------------------------------------------------
 * Batched solver: many independent SPD systems in one persistent launch.  The reference
 * solves one system per launch (host/cuper_control_xrt_host.cpp:205-272, one
 * cuper_pcg_control_kernel run per dataset); a caller with many systems looped over
 * CsrDataset::load + run.  Here all systems are resident at once and thread-block clusters
 * take them from a device work queue, largest first.  Each system follows the single-system
 * iteration (row-sum form, FP32 vectors, FP64 solution and FP64 residual replacement) and
 * gets its own status / iterations / FP64 true residual.  Vectors b and x are the systems'
 * vectors concatenated in the order they were given, each in its original row order.
 * ------------------------------------------------------------------------------------ */
typedef struct xplus_batch xplus_batch;

/* nsys systems, system k given as CSR (row_ptrs[k][ns[k]+1], col_idxs[k], values[k], FP64).
 * opts: value_type F32 | BF16 | F16, vector_type F32, sigma, chunk, index16, replace_drop,
 * replace_every, restart_on_replace, stagnation_gain, stagnation_window, split_ratio, device;
 * the others are ignored.  The launch shape starts
 * at clusters of 4 CTAs x 512 threads (xplus_batch_set_launch / xplus_batch_autotune). */
int xplus_batch_create(int nsys, const int* const* row_ptrs, const int* const* col_idxs,
                       const double* const* values, const int* ns, const xplus_opts* opts,
                       xplus_batch** out);
int xplus_batch_destroy(xplus_batch* h);
/* cluster in {1, 2, 4, 8} CTAs, block_threads in {128, 256, 512}; the grid is as many
 * clusters as the device holds at once.  XPLUS_ERR_CUDA when the shape cannot launch. */
int xplus_batch_set_launch(xplus_batch* h, int cluster, int block_threads);
/* The `count` largest systems (by nnz * sqrt(n)) in a launch of their own, concurrent with the
 * launch of the rest on a second stream, with clusters of `cluster` CTAs in {4, 8, 16} (16 is
 * beyond the portable limit, allowed on B200) of block_threads threads, one cluster per system;
 * count 0: one launch for all.  No wait spans two clusters, so the two launches need no
 * co-residency; the largest system, which otherwise runs on a main-launch cluster for the
 * whole makespan, gets up to 16 SMs.  XPLUS_ERR_CUDA when the shape cannot launch. */
int xplus_batch_set_split(xplus_batch* h, int count, int cluster, int block_threads);
/* The current split: count (0: none), cluster, block_threads and grid of its launch. */
int xplus_batch_split_info(xplus_batch* h, int* count, int* cluster, int* block_threads, int* grid);
/* on != 0: both launches run the cluster-resident kernel.  Each CTA of a cluster keeps, for the
 * whole solve of its system, its band's r, Ap', dx, M^-1 and row sums and the window of the
 * search direction that its columns reach in shared memory (the single-system SM-resident
 * iteration with one cluster barrier per iteration); each launch is given the dynamic shared
 * memory of the largest band among the systems it takes.  XPLUS_ERR_ARG when a system does not
 * fit at its launch's cluster size (split the largest systems off into bigger clusters first);
 * 0: the global-memory kernel (two cluster barriers per iteration, no shared-memory limit). */
int xplus_batch_set_resident(xplus_batch* h, int on);
/* Whether the resident kernel is on, and the dynamic shared memory (bytes per CTA) of the main
 * and the split launch (0 when off or no split). */
int xplus_batch_resident_info(xplus_batch* h, int* on, int* smem, int* smem_split);
/* on != 0 (the default): each resident launch is given the most dynamic shared memory that
 * keeps its occupancy (all a CTA may have, or half an SM's when two CTAs share one), and a CTA
 * whose band's matrix (values and columns) fits beside its vectors copies it there once per
 * system; its SpMV then reads no global memory.  Same products in the same order, so the
 * results are the same bit for bit.  0: every launch sized to its largest band, the matrix
 * read from global memory. */
int xplus_batch_set_stage_matrix(xplus_batch* h, int on);
/* Whether matrix staging is on, and over the last resident solve the systems whose every CTA
 * staged its band's matrix (systems_all) and those where only some did (systems_some); both 0
 * with the global-memory kernel. */
int xplus_batch_staged_info(xplus_batch* h, int* on, int* systems_all, int* systems_some);
/* The launch-shape autotuner: times every cluster x block_threads shape that launches and keeps
 * the fastest, with x0 = 0 for every system; then, on that shape, splits off the 1, 2, 4, 8 or
 * 16 largest systems (at most a quarter of them) into clusters of 16 x 512, 8 x 512 or 16 x 256;
 * then the resident kernel, with main launches of 2, 4 or 8 CTAs x 256 or 512 threads and the
 * systems that do not fit the main launch's shared memory (or half an SM's, so that two CTAs
 * share one) in a split launch of 16-CTA clusters.  It keeps the fastest of all
 * (xplus_batch_split_info and xplus_batch_resident_info report it).  iters > 0: that many
 * PCG iterations per system on b = 1; iters <= 0: every system solved to FP64 true relative
 * residual tau (0 < tau < 1) on the right-hand side of the last solve (b = 1 before any solve),
 * so the queue's makespan on the caller's workload is what is timed.  Returns the main shape
 * and the best time (min of 2 runs). */
int xplus_batch_autotune(xplus_batch* h, int iters, double tau, int* cluster, int* block_threads,
                         double* best_ms);
/* Blocking solve with host vectors of length sum(ns) (x0 NULL: zeros).  tau / tau_mode /
 * max_iters as xplus_pcg_solve, applied to every system (relative tolerances per system). */
int xplus_batch_solve(xplus_batch* h, const double* b, const double* x0, double tau, int tau_mode,
                      int max_iters, double* x_out);
/* Asynchronous solve on device vectors (d_x: x0 in, x out) enqueued on `stream` (NULL: the
 * handle's stream) as one CUDA graph (gather, persistent launch, scatter).  The graph is
 * captured on the first call and replayed while d_b, d_x, tau, tau_mode, max_iters and the
 * launch shape stay the same.  d_b and d_x must be device (or managed) memory of the
 * handle's GPU: host or other-GPU pointers return XPLUS_ERR_ARG before anything is enqueued. */
int xplus_batch_solve_device(xplus_batch* h, const double* d_b, double* d_x, double tau, int tau_mode,
                             int max_iters, void* stream);
/* Outcome of the last solve, per system (each array nullable, nsys long): status, inner
 * iterations, FP64 residual replacements, FP64 true relative residual, device time from the
 * system's start to its end; kernel_ms: device time of the whole solve. */
int xplus_batch_results(xplus_batch* h, int* status, int* iterations, int* replacements, double* true_rel,
                        double* system_ms, double* kernel_ms);
/* Total rows and stored nonzeros, launch shape, and the bytes one SpMV over every system
 * moves in the stored format (off-diagonal value + index, row sums, x read, y written). */
int xplus_batch_info(xplus_batch* h, int64_t* total_n, int64_t* total_nnz, int* cluster, int* block_threads,
                     int* grid, int64_t* spmv_bytes);

/* ------------------------------------------------------------------------------------
 * Multi-kernel ABI: the five "kernel functions" of archived/include/cg_kernels.hpp:9-54
 * with the same names and arguments, run on the GPU.  Pointers may be device pointers
 * (zero copy) or plain host pointers (staged through device buffers), so the reference's
 * run_local_multi_kernel_solver (archived/host/multi_kernel_solver.hpp:100) can link
 * against this library unchanged.  There is no n <= 1024 cap; n < 0 returns silently
 * as valid_n() does (archived/kernels/cg_kernels.cpp:9-12).  Each call is blocking.
 * ------------------------------------------------------------------------------------ */
void spmv_csr_kernel(const int* row_ptr, const int* col_idx, const double* values,
                     const double* x, double* y, int n);
void spmv_blocked_kernel(const int* row_ptr, const int* col_idx, const double* values,
                         const double* x, double* y, int n);
void init_pcg_kernel(const double* b, const double* ax, const double* m_inv, double* r,
                     double* z, double* p, double* metrics, int n);
void dot_kernel(const double* a, const double* b, double* out, int n);
void update_xrz_kernel(double* x, const double* p, double* r, const double* ap,
                       const double* m_inv, double* z, double* metrics, double alpha, int n);
void update_p_kernel(const double* z, double* p, double beta, int n);

/* No-allocation variant of update_xrz_kernel.  It has no counterpart in the reference.
 *
 * Some callers cannot call cudaMalloc: code that runs inside another framework's fixed
 * device-memory budget, or a latency-critical loop where an allocation (which can
 * synchronize the device, or fail under memory pressure) is not allowed.  This entry point
 * allocates nothing.  Its only scratch, one FP64 pair per reduction block, is a 16 KiB array
 * compiled into the library, which every GPU that loads the library holds until the process
 * exits.  The caller still passes every input and output, as device pointers: x, r, z are
 * updated as update_xrz_kernel updates them, and metrics[0..1] = {r.z, r.r} is written on
 * the device.  The call is asynchronous on `stream` (a cudaStream_t; NULL = the legacy
 * default stream).
 *   - Every pointer must be device memory of the current device (or managed memory).
 *     Host arrays, which update_xrz_kernel accepts and stages, and another GPU's memory
 *     return XPLUS_ERR_ARG with a message before anything is launched.
 *   - The first call on each device looks the scratch array's device address up with
 *     cudaGetSymbolAddress (again after the device's context was reset); make that first
 *     call before any stream capture.
 *   - An error left pending on the calling thread by earlier asynchronous work is reported
 *     as XPLUS_ERR_CUDA, left in place for its owner, and nothing is launched.
 *   - All calls share the one scratch array, which keeps the last call's contents: calls
 *     that overlap on the GPU (other streams, other host threads) race; serialize them.
 *   - n may be at most XPLUS_NOALLOC_MAX_N (1024 reduction blocks x 256 threads x 16
 *     elements); a larger n returns XPLUS_ERR_ARG with a message and launches nothing. */
#define XPLUS_NOALLOC_MAX_N 4194304
int xplus_update_xrz_noalloc(double* x, const double* p, double* r, const double* ap,
                             const double* m_inv, double* z, double* metrics, double alpha, int n,
                             void* stream);

/* ------------------------------------------------------------------------------------
 * Host-side data path (no GPU needed).
 * ------------------------------------------------------------------------------------ */

/* CsrDataset::load: reads row_ptr.txt col_idx.txt values.txt b.txt x0.txt from dir with
 * the same validation and messages.  Two-phase: call with NULL arrays to get n, nnz. */
int xplus_dataset_load_text(const char* dir, int* n, int* nnz, int* row_ptr, int* col_idx,
                            double* values, double* b, double* x0);
/* Binary cache of the same five arrays (one file).  Same two-phase protocol. */
int xplus_dataset_save_binary(const char* path, int n, int nnz, const int* row_ptr,
                              const int* col_idx, const double* values, const double* b,
                              const double* x0);
int xplus_dataset_load_binary(const char* path, int* n, int* nnz, int* row_ptr, int* col_idx,
                              double* values, double* b, double* x0);

/* extract_jacobi_diag: XPLUS_ERR_DATA with the reference's message on a missing/zero entry. */
int xplus_jacobi_diag(int n, const int* row_ptr, const int* col_idx, const double* values,
                      double* diag);

/* Synthetic SPD systems.  Two-phase: out arrays NULL -> *n, *nnz.  The matrix is the
 * P1 finite-element stiffness matrix of -div(k grad u) on the unit square (cube) with
 * interior nodes g x g (x g), jittered nodes, log-normal per-element conductivity and
 * eliminated Dirichlet boundary.  perm_seed >= 0 applies a seeded random symmetric
 * permutation; rcm != 0 then applies reverse Cuthill-McKee.  x_true ~ U(-1,1) from
 * x_seed, b = A x_true (FP64), x0 = 0. */
int xplus_gen_fem2d(int g, double sigma, double jitter, uint64_t seed, int64_t perm_seed,
                    int rcm, uint64_t x_seed, int* n, int* nnz, int* row_ptr, int* col_idx,
                    double* values, double* b, double* x_true);
int xplus_gen_fem3d(int g, double sigma, double jitter, uint64_t seed, int64_t perm_seed,
                    int rcm, uint64_t x_seed, int* n, int* nnz, int* row_ptr, int* col_idx,
                    double* values, double* b, double* x_true);

/* Reverse Cuthill-McKee ordering of a structurally symmetric CSR: perm[new] = old. */
int xplus_rcm(int n, const int* row_ptr, const int* col_idx, int* perm);
/* The same reverse Cuthill-McKee ordering computed on the GPU from a device CSR, bit-identical
 * to xplus_rcm: one cooperative launch per BFS builds the Cuthill-McKee levels in parallel
 * (each node of the next level goes to its lowest-positioned neighbour in the current level,
 * each parent's children ordered by (degree, index)), the pseudo-peripheral search and the
 * component order as xplus_rcm has them.  A graph it does not cover (a node with more than 64
 * children in one level, or a repeated column in a row) is ordered by the host function instead,
 * with the same result; *used_gpu (nullable) says which ran.  Device pointers of the current
 * GPU; blocks until d_perm is written.  No reference counterpart (the reference orders on the
 * host while packing, host/cuper_control_matrix.hpp:130-207). */
int xplus_rcm_device(int n, const int* d_row_ptr, const int* d_col_idx, int* d_perm, int* used_gpu, void* stream);
/* B = P A P^T for perm[new] = old (columns sorted ascending in each output row). */
int xplus_permute_symmetric(int n, const int* row_ptr, const int* col_idx, const double* values,
                            const int* perm, int* out_row_ptr, int* out_col_idx,
                            double* out_values);
/* xplus_permute_symmetric on device arrays (thread per output row, stable ordering of the
 * renumbered columns), bit-identical to it; blocks until the outputs are written. */
int xplus_permute_symmetric_device(int n, const int* d_row_ptr, const int* d_col_idx, const double* d_values,
                                   const int* d_perm, int* d_out_row_ptr, int* d_out_col_idx,
                                   double* d_out_values, void* stream);

/* SELL-C-sigma layout (host builder; the device copies come from the same function).
 * Two-phase: pass NULL outputs to get n_slices, slots.  perm[new] = old row,
 * slice_ptr[n_slices+1] (in slots), slice_width[n_slices], col[slots] in new numbering,
 * val[slots] (FP64).  diag_split != 0 leaves the diagonal out (returned in diag[n],
 * new order).  Padding slots hold col = own row, val = 0. */
int xplus_sell_build(int n, const int* row_ptr, const int* col_idx, const double* values,
                     int C, int sigma, int chunk, int diag_split, int* n_slices, int64_t* slots,
                     int* perm, int64_t* slice_ptr, int* slice_width, int* col, double* val,
                     double* diag);

/* The same SELL-C-sigma layout built on the GPU from device CSR arrays, bit-identical to
 * xplus_sell_build (C = 32, sigma <= 4096).  Two-phase: NULL d_col, d_val and d_diag return
 * only *n_slices and *slots (d_perm, d_slice_ptr, d_slice_width are filled when given).
 * Outputs are device arrays of the sizes xplus_sell_build uses (d_diag: n).  Temporaries are
 * allocated and freed inside; the call returns after the work on `stream` is done. */
int xplus_sell_build_device(int n, const int* d_row_ptr, const int* d_col_idx, const double* d_values,
                            int C, int sigma, int chunk, int diag_split, int* n_slices, int64_t* slots,
                            int* d_perm, int64_t* d_slice_ptr, int* d_slice_width, int* d_col,
                            double* d_val, double* d_diag, void* stream);

/* Cuper packed-format import (host/cuper_control_matrix.hpp:73-83,130-207): decode the
 * 16 channel streams (channel_words words each) into COO triplets in the order they are
 * stored, skipping padding.  Returns the count in *nnz_out; rows/cols/vals may be NULL
 * for a size query. */
int xplus_cuper_unpack(int n, int batch_count, const int* sp_element_list_ptr,
                       const uint64_t* words, int64_t channel_words, int64_t* nnz_out,
                       int* rows, int* cols, float* vals);

#ifdef __cplusplus
}
#endif

#endif /* XPLUS_B200_H */
