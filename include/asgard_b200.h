/* asgard_b200 -- C ABI of the B200 (sm_100a) kronmult operator and the
 * implicit backward-Euler GMRES solve it feeds.
 *
 * Plain pointers and sizes only; every entry point returns an asgk_status
 * (0 = success) and never throws.  Device pointers are CUDA global-memory
 * pointers on the current device; "host" pointers are ordinary host memory.
 * A plan is not re-entrant: one call at a time per plan, as with the
 * reference's kronmult_matrix::apply, which is documented "not thread-safe"
 * (src/asgard_kronmult_matrix.hpp:336).  Calls are stream-ordered on the
 * stream argument (0 = the legacy default stream).
 *
 * Conventions shared with the reference (src/device/asgard_kronmult.hpp):
 *   - a Kronecker product acts on tensors of n^d entries stored contiguously,
 *     dimension 0 slowest;
 *   - the d factors of one product are column-major n x n blocks inside vA,
 *     addressed by iA offsets, the first offset applying to dimension 0;
 *   - y = beta*y + alpha * sum_{pairs (row,col)} sum_{terms}
 *           (A_{t,0} (x) ... (x) A_{t,d-1}) x_col, with beta = 0 overwriting y.
 */
#ifndef ASGARD_B200_H
#define ASGARD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct asgk_plan asgk_plan;
typedef struct asgk_mlp asgk_mlp;
typedef struct asgk_jacobi asgk_jacobi;
typedef void *asgk_stream; /* a cudaStream_t */

typedef enum asgk_status
{
  ASGK_OK              = 0,
  ASGK_ERR_INVALID     = 1, /* bad argument (size, pointer, index) */
  ASGK_ERR_UNSUPPORTED = 2, /* (d, n) outside the supported range */
  ASGK_ERR_CUDA        = 3, /* a CUDA runtime call failed */
  ASGK_ERR_ALLOC       = 4, /* device or host allocation failed */
  ASGK_ERR_BREAKDOWN   = 5, /* GMRES: zero or non-finite Arnoldi norm */
  ASGK_ERR_NOT_CONVERGED = 6, /* GMRES: iteration limit before tolerance */
  ASGK_ERR_NONFINITE   = 7, /* non-finite residual (NaN/Inf in the data) */
  ASGK_ERR_NOALLOC_LIMIT = 8, /* request exceeds an allocation-free entry's fixed scratch */
  ASGK_ERR_DEVICE_TIMEOUT = 9 /* a kernel's bounded wait on its own copies expired;
                                 the outputs of that launch are invalid */
} asgk_status;

typedef enum asgk_precision
{
  ASGK_FP64 = 0, /* FP64 loads, FP64 arithmetic */
  ASGK_FP32 = 1, /* FP64 vectors, FP32 factors and FP32 arithmetic */
  ASGK_BF16 = 2  /* FP64 vectors, BF16 tensor-core products, FP32 accumulation */
} asgk_precision;

/* ---------------------------------------------------------------- plans */

/* Replaces kronmult_matrix<P>'s sparse constructors
 * (src/asgard_kronmult_matrix.hpp:235-297, CPU one-call and multi-call forms)
 * and the buffers make_kronmult_sparse uploads
 * (src/asgard_kronmult_matrix.cpp:639-643).
 *
 * row_ptr[num_rows+1], col_indx[nnz]: pairs in CSR form over output cells
 *   (the reference's CPU format); col_indx are cell indices < num_cols.
 * iA[nnz*num_terms*d]: offsets into vA of the n x n factors, pair-major then
 *   term then dimension (reference layout).
 * vA[vA_len]: factor values (FP64, host).
 * All arrays are host arrays and are copied; the plan owns device copies.
 * Offsets are checked against vA_len (ASGK_ERR_INVALID if out of range). */
int asgk_plan_create(asgk_plan **plan, int d, int n, int num_rows,
                     int num_cols, int num_terms, const int64_t *row_ptr,
                     const int *col_indx, const int *iA, const double *vA,
                     int64_t vA_len);

/* Same operator from the reference's GPU pair format (kronmult::gpu_sparse,
 * src/device/asgard_kronmult.hpp:113-133): per pair the tensor offsets
 * iy[i] (into y) and ix[i] (into x), both multiples of n^d, any order.
 * Pairs are grouped by output cell inside the plan. */
int asgk_plan_create_pairs(asgk_plan **plan, int d, int n, int num_rows,
                           int num_cols, int num_terms, int64_t num_batch,
                           const int *iy, const int *ix, const int *iA,
                           const double *vA, int64_t vA_len);

/* Sparse-grid form used by the builder below: per pair the d 1D connection
 * indices conn[nnz*d]; factor (t, k) of a pair is the n x n block at
 * vA + conn[k]*(d*T*n*n) + (t*d + k)*n*n (the layout make_kronmult_sparse
 * writes, src/asgard_kronmult_matrix.cpp:369-393, 455-461) -- this stores
 * d indices per pair instead of d*T. */
int asgk_plan_create_conn(asgk_plan **plan, int d, int n, int num_rows,
                          int num_cols, int num_terms, const int64_t *row_ptr,
                          const int *col_indx, const int *conn,
                          const double *vA, int64_t vA_len);

/* The sparse-grid operator with its connected pairs found on the device:
 * the element table of dimension d and level `level` (asgk_sparse_grid),
 * every cell pair tested against the 1D connectivity (the reference's
 * check_connected rule, src/asgard_kronmult_matrix.cpp:230-300, which
 * make_kronmult_sparse applies on the host, :406-466) by a kernel, the pair
 * list written straight into the plan.  vA in the per-1D-connection layout
 * of asgk_plan_create_conn.  The same plan as asgk_build_pairs followed by
 * asgk_plan_create_conn (the same pairs in the same order), without the
 * host pass and the copy of the pair list. */
int asgk_plan_create_grid(asgk_plan **plan, int d, int n, int level,
                          int num_terms, const double *vA, int64_t vA_len);

/* Dense form: replaces kronmult_matrix<P>'s dense constructor
 * (src/asgard_kronmult_matrix.hpp:132-176, filled by make_kronmult_dense,
 * src/asgard_kronmult_matrix.cpp:64-163) and kronmult::gpu_dense /
 * cpu_dense (src/device/asgard_kronmult.hpp:81-125,
 * src/device/asgard_kronmult_cpu.cpp:160-530): every output cell r <
 * num_rows with every input cell c < num_cols,
 *   y_r = beta y_r + alpha sum_c sum_t (A_{t,0} (x) ... (x) A_{t,d-1}) x_c,
 * A_{t,k} the n x n column-major block of terms[t] at
 *   terms[t] + ((k*num_1d_blocks + ic)*num_1d_blocks + ir)*n*n,
 * ir = elem[(r + row_offset)*d + k], ic = elem[(c + col_offset)*d + k]
 * (1D cell indices < num_1d_blocks).
 * terms[num_terms]: host arrays of d*num_1d_blocks^2*n^2 values each;
 * elem[elem_len]: host array, elem_len >= d*(max(row_offset + num_rows,
 * col_offset + num_cols)).  num_terms == 0 makes the reference's empty
 * matrix (apply only scales y).  The plan holds every (row, col) pair (the
 * reference's num_batch() = rows*cols products per apply).  Indices out of
 * range: ASGK_ERR_INVALID. */
int asgk_plan_create_dense(asgk_plan **plan, int d, int n, int num_rows,
                           int num_cols, int num_terms,
                           const double *const *terms, const int *elem,
                           int64_t elem_len, int row_offset, int col_offset,
                           int num_1d_blocks);

/* Replaces kronmult_matrix<P>::set_workspace
 * (src/asgard_kronmult_matrix.hpp:301-307): device buffers of at least
 * input_size / output_size doubles that asgk_apply_host stages x and y in
 * (the caller keeps them alive and may share them between plans that are
 * not applied at the same time).  Without it a plan allocates its own on
 * its first host apply. */
int asgk_plan_set_workspace(asgk_plan *plan, double *x, int64_t x_len,
                            double *y, int64_t y_len);

/* What kind of plan this is: 0 sparse (pair list), 1 dense, 2 global
 * Kronecker form; negative on a null plan.  kronmult_matrix::is_dense()
 * (src/asgard_kronmult_matrix.hpp:514-517) is kind == 1. */
int asgk_plan_kind(const asgk_plan *plan);

/* Global Kronecker form (the reference's global_kron_matrix,
 * src/asgard_kronmult_matrix.cpp:1196-1334, and global_cpu,
 * src/device/asgard_glkronmult_cpu.cpp:103-181): the same operator as the
 * connected-pair plan of this sparse grid (the element table `table`,
 * num_cells x 2d, as asgk_sparse_grid writes it; vA in the per-1D-connection
 * layout of asgk_plan_create_conn), applied through the cell pairs that
 * differ in at most one dimension.  A term that is the identity
 * (self-connection blocks I, all others 0) in all dimensions but one is
 * applied in one pass with the others; a term acting in m >= 2 dimensions
 * as the reference does it: 2^(m-1) chains of m 1D passes over the upper or
 * lower parts of its 1D operators (its permutes), summed.  n = 3 only.  The
 * plan works with asgk_apply / asgk_apply_euler / the GMRES and Jacobi
 * entries like any other; asgk_plan_info's num_batch reports the neighbour
 * entries one apply visits and flops 2 * n^(d+1) per entry.
 * asgk_plan_update_values keeps the dimensions each term acts in
 * (ASGK_ERR_INVALID if they change). */
int asgk_plan_create_global(asgk_plan **plan, int d, int n, int level,
                            int num_cells, const int *table, int num_terms,
                            const double *vA, int64_t vA_len);
void asgk_plan_destroy(asgk_plan *plan);

/* Replaces update_stored_coefficients (src/asgard_kronmult_matrix.hpp:519-536):
 * vA in the layout the plan was created with (same length).  For a dense
 * plan use asgk_plan_update_terms. */
int asgk_plan_update_values(asgk_plan *plan, const double *vA, int64_t vA_len);

/* Dense plans: replaces the per-term overload of update_stored_coefficients
 * (src/asgard_kronmult_matrix.hpp:538-561); terms[num_terms] as for
 * asgk_plan_create_dense.  ASGK_ERR_INVALID on other plans. */
int asgk_plan_update_terms(asgk_plan *plan, const double *const *terms,
                           int num_terms);

/* Sizes: tensor_size = n^d, input_size = num_cols*n^d,
 * output_size = num_rows*n^d, num_batch = the (row, col) products one apply
 * computes (nnz; rows*cols for a dense plan), flops = 2*d*T*n^(d+1)*num_batch
 * (compute_flops, src/asgard_kronmult_matrix.hpp:507-512). */
int asgk_plan_info(const asgk_plan *plan, int64_t *num_batch,
                   int64_t *input_size, int64_t *output_size,
                   int64_t *flops, int64_t *device_bytes);

/* ---------------------------------------------------------------- apply */

/* y = beta*y + alpha*K*x on device pointers
 * (kronmult_matrix<P>::apply<resource::device>, src/asgard_kronmult_matrix.hpp:340-478).
 * precision selects the arithmetic; x and y are FP64. */
int asgk_apply(asgk_plan *plan, int precision, double alpha, const double *x,
               double beta, double *y, asgk_stream stream);

/* FP32 vectors: y = beta*y + alpha*K*x with FP32 x, y and arithmetic
 * (kronmult_matrix<float>::apply<resource::device>). */
int asgk_apply_f32(asgk_plan *plan, float alpha, const float *x, float beta,
                   float *y, asgk_stream stream);

/* Host pointers: copies x (and y when beta != 0) to the plan's device
 * workspace, applies in FP64 and copies y back, synchronising the stream
 * (kronmult_matrix<P>::apply<resource::host> on a CUDA build,
 * src/asgard_kronmult_matrix.hpp:351-358, 451-452). */
int asgk_apply_host(asgk_plan *plan, double alpha, const double *x,
                    double beta, double *y, asgk_stream stream);

/* The backward-Euler operator of simple_gmres_euler (src/solver.cpp:119-135)
 * fused into one pass: y = beta*y + alpha*(x - dt*K*x).  Square plans only. */
int asgk_apply_euler(asgk_plan *plan, int precision, double dt, double alpha,
                     const double *x, double beta, double *y,
                     asgk_stream stream);

/* ---------------------------------------------------------------- GMRES */

typedef struct asgk_gmres_info
{
  double error;       /* final residual estimate (as the reference reports) */
  int iterations;     /* reference count: 1 per restart + 1 per Arnoldi step */
  int status;         /* asgk_status of the solve */
  double true_relres; /* ||b - (I - dt K) x||_2 / ||b||_2 recomputed in FP64 */
  int outer_steps;    /* refinement steps (mixed precision), else restarts */
  int matvecs_low;    /* low-precision operator applications */
  int matvecs_fp64;   /* FP64 operator applications */
  int precond_calls;  /* preconditioner applications */
  int fallback;       /* 1 if the learned preconditioner was dropped */
} asgk_gmres_info;

typedef enum asgk_tol_mode
{
  ASGK_TOL_ABS = 0, /* reference semantics: |s_k g_k| <= tol (src/solver.cpp:258-259) */
  ASGK_TOL_REL = 1  /* residual <= tol * ||b||_2 */
} asgk_tol_mode;

/* Solves (I - dt*K) x = b on device vectors, x holding the initial guess.
 * Replaces solver::simple_gmres_euler (src/solver.hpp:34-40,
 * src/solver.cpp:119-135 and the template :157-298) with a device-resident
 * GMRES: classical Gram-Schmidt, Givens rotations, packed Hessenberg.
 *
 * precision = ASGK_FP64 is the reference algorithm.  ASGK_FP32/ASGK_BF16 run
 * the Krylov operator in that arithmetic inside FP64 iterative refinement
 * (outer FP64 residuals; FP64 Gram-Schmidt, norms and least squares), until
 * the FP64 residual meets tol.
 * precond: a learned preconditioner (asgk_mlp) applied on the right through
 * flexible GMRES, or NULL.  restart <= 0 selects default_gmres_restarts
 * (src/solver.cpp:142-152); max_outer <= 0 selects n. */
int asgk_gmres_euler(asgk_plan *plan, double dt, double *x, const double *b,
                     int restart, int max_outer, double tol, int tol_mode,
                     int precision, asgk_mlp *precond, asgk_gmres_info *info,
                     asgk_stream stream);

/* solver::simple_gmres on a dense column-major n x n host matrix (the test
 * path of src/solver.cpp:55-74) with an empty M: no preconditioner; the same
 * as asgk_gmres_dense_precond with M = NULL. */
int asgk_gmres_dense(int n, const double *A, double *x, const double *b,
                     int restart, int max_outer, double tol,
                     asgk_gmres_info *info);
/* simple_gmres_euler of kronmult_matrix<float> (the reference's FP32
 * instantiation, src/solver.cpp:119-135 with P = float,
 * src/asgard_kronmult_matrix.cpp:1633): x (initial guess and result) and b
 * are FP32 device vectors.  The solve runs on FP64 copies of them (allocated
 * for the call) with the FP32 operator inside FP64 iterative refinement,
 * stopping when the FP64 residual ||b - (I - dt K) x|| is at most tol (the
 * reference's absolute criterion; tol <= 0 selects its FP32 default 1e-6),
 * and x is rounded back to FP32.  Synchronises the stream. */
int asgk_gmres_euler_f32(asgk_plan *plan, float dt, float *x, const float *b,
                         int restart, int max_outer, float tol,
                         asgk_gmres_info *info, asgk_stream stream);

/* simple_gmres(A, x, b, M, restart, max_iter, tol) with the reference's
 * dense preconditioner M (src/solver.cpp:11-38, 55-74): M (column-major
 * host n x n, or NULL for none) is LU-factored with partial pivoting and
 * applied on the left to the residual and to every new basis vector, so the
 * tolerance is on the estimated preconditioned residual, as in the
 * reference.  A singular M: ASGK_ERR_BREAKDOWN before any device work. */
int asgk_gmres_dense_precond(int n, const double *A, double *x,
                             const double *b, const double *M, int restart,
                             int max_outer, double tol, asgk_gmres_info *info);

/* One classical Gram-Schmidt step of the device GMRES, the two GEMVs and the
 * norm of src/solver.cpp:233-245:
 *   h[0..k) = V[:, 0..k)^T w;   w -= V[:, 0..k) h;   *norm = ||w||_2.
 * V is column-major with leading dimension ldv >= n; V, w and h are device
 * pointers, norm a host pointer.  Deterministic (fixed-order reductions).
 * The partial sums live in scratch allocated on the stream for the call. */
int asgk_cgs_step(const double *V, int64_t ldv, int k, double *w, int64_t n,
                  double *h, double *norm, asgk_stream stream);

/* asgk_cgs_step without any device allocation, for callers that must not
 * allocate once their solve runs (all device memory handed to their own pool
 * at start-up, or no device-wide synchronisation allowed).  No counterpart in
 * the reference.  Same arguments and result as asgk_cgs_step; the partial
 * sums use a fixed array of 1 MiB inside the library (held on every
 * GPU that loads it until exit).  k <= 256 columns and at most 512 reduction
 * blocks (GPUs up to 256 SMs), else ASGK_ERR_NOALLOC_LIMIT.  All calls share
 * the array: calls that overlap on the GPU race.  The first call on a device
 * looks up the array's address (make it before any stream capture). */
int asgk_cgs_step_noalloc(const double *V, int64_t ldv, int k, double *w,
                          int64_t n, double *h, double *norm,
                          asgk_stream stream);

/* default_gmres_restarts<double>(n) (src/solver.cpp:142-152). */
int asgk_default_gmres_restarts(int64_t n);

/* ------------------------------------------------ Jacobi preconditioners */

typedef enum asgk_jacobi_kind
{
  ASGK_JACOBI_POINT = 0, /* the reference's diagonal preconditioner */
  ASGK_JACOBI_BLOCK = 1, /* inverse of each cell's n^d x n^d diagonal block */
  ASGK_JACOBI_KRON  = 2, /* the same inverse through the eigendecompositions of
                            the block's 1D factors (global plans whose terms act
                            in one dimension each; any d <= 6) */
  ASGK_JACOBI_LINE  = 3  /* no counterpart in the reference: exact solves along
                            the pencils of every dimension whose 1D operator is
                            symmetric (1 to 3 such dimensions), chained
                            M_km^-1 B ... B M_k1^-1 with B the cell-diagonal
                            part of those dimensions' terms; global plans whose
                            terms act in one dimension each, n = 3, d <= 6;
                            ASGK_ERR_UNSUPPORTED without such a dimension */
} asgk_jacobi_kind;

/* Builds a Jacobi preconditioner of I - dt*K for a square plan, on the
 * device.  ASGK_JACOBI_POINT is build_preconditioner
 * (src/asgard_kronmult_matrix.cpp:1015-1067): pc_i = sum_t prod_k
 * A_{t,k}(i_k, i_k) over the factors of each cell's own pair, applied as
 * z_i = v_i / (1 - dt*pc_i) (apply_diagonal_precond, src/solver.cpp:76-91;
 * the reference has it in its global-kron mode only).  ASGK_JACOBI_BLOCK
 * inverts the whole diagonal block (I - dt*sum_t (x)_k A_{t,k}) of every
 * cell (Gauss-Jordan with partial pivoting; n^d <= 81, else
 * ASGK_ERR_UNSUPPORTED); ASGK_ERR_BREAKDOWN if a block is singular.
 * ASGK_JACOBI_KRON applies the block inverse of a global plan whose terms
 * act in one dimension each (there the block is a Kronecker sum of the
 * cell's 3x3 self blocks): each 3x3 factor is diagonalised on the host and
 * the inverse applied as 2d complex contractions per cell, O(d n^(d+1))
 * work and a few hundred bytes of tables per cell; ASGK_ERR_UNSUPPORTED for
 * other plans or a factor that is defective or badly conditioned.  The
 * preconditioner keeps no reference to the plan. */
int asgk_jacobi_create(asgk_jacobi **pc, asgk_plan *plan, double dt, int kind);
void asgk_jacobi_destroy(asgk_jacobi *pc);
/* z = M v on device vectors of the plan's size (z != v). */
int asgk_jacobi_apply(asgk_jacobi *pc, const double *v, double *z,
                      asgk_stream stream);
/* z = M v as the solves of the given precision apply it: ASGK_FP64 as
 * asgk_jacobi_apply, ASGK_FP32 in the FP32 arithmetic (FP16 block inverses
 * for ASGK_JACOBI_BLOCK) of the FP32 inner solves of asgk_gmres_euler_jacobi.
 * No counterpart in the reference (its diagonal preconditioner has one
 * precision). */
int asgk_jacobi_apply_precision(asgk_jacobi *pc, int precision,
                                const double *v, double *z, asgk_stream stream);
int asgk_jacobi_info(asgk_jacobi *pc, int *kind, double *dt,
                     int64_t *device_bytes);
/* asgk_gmres_euler with a Jacobi preconditioner applied on the right
 * (flexible GMRES; the reference applies its diagonal one to the residual).
 * With ASGK_FP32 the block inverses are applied from an FP16 copy (FP64
 * accumulation): an inexact preconditioner, which flexible GMRES allows.
 * A preconditioner built on a plan of another shape (cells or n^d) is
 * refused with ASGK_ERR_INVALID before any launch. */
int asgk_gmres_euler_jacobi(asgk_plan *plan, double dt, double *x,
                            const double *b, int restart, int max_outer,
                            double tol, int tol_mode, int precision,
                            asgk_jacobi *precond, asgk_gmres_info *info,
                            asgk_stream stream);

/* Restart cycles of the device GMRES run as recorded CUDA graphs (one
 * launch per cycle: each Arnoldi step's Givens update runs on the device,
 * writes the cycle's go flag and, at the end of a graph node, opens the next
 * node, so no host round trip per iteration) whenever the preconditioner is
 * none or Jacobi; the host-driven loop otherwise, or with enable = 0.  Both
 * give the same iterates bit for bit.  Process-wide; returns the previous
 * setting.  No counterpart in the reference. */
int asgk_set_gmres_graphs(int enable);

/* Arnoldi steps per conditional node of a recorded cycle (default 16) for
 * plans whose step kernels can skip themselves (global plans whose terms act
 * in one dimension each, with a Jacobi preconditioner or none; one step per
 * node otherwise).  Inside a node, the kernels of the steps after the cycle
 * stopped return at once; iterates are the same for every value.  steps < 1
 * only reads the setting.  Process-wide; returns the previous setting. */
int asgk_set_gmres_node_steps(int steps);

/* The FP32 inner solves of iterative refinement (precision ASGK_FP32) run
 * their Gram-Schmidt passes over an FP32 copy of the Krylov basis (fp32 = 1,
 * the default): each new basis vector is normalised in FP64 and also stored
 * rounded to FP32, and the projections h = V^T w and the update w -= V h
 * read that copy, with w, h and every sum in FP64.  The operator, the
 * preconditioner and the solution update keep the FP64 vectors, and the
 * outer FP64 residual decides convergence as before.  fp32 = 0 reads the
 * FP64 basis.  Process-wide; returns the previous setting.  No counterpart
 * in the reference. */
int asgk_set_gmres_basis(int fp32);

/* Solves with the line preconditioner and the FP32 global operator at
 * d >= 5 (asgk_gmres_euler_jacobi): with on = 1 (the default) the
 * preconditioner's last pass also writes the FP32 copy of its output that
 * the operator reads, instead of a separate conversion pass over the vector;
 * on = 0 keeps the separate pass.  Both give the same bits.  Process-wide;
 * returns the previous setting.  No counterpart in the reference. */
int asgk_set_gmres_fused_copy(int on);

/* Relative tolerance of each inner solve of iterative refinement with the
 * BF16 tensor-core operator (precision ASGK_BF16; default 1e-3): the
 * operator's products use BF16-rounded operands (relative rounding 2^-9), so
 * every refinement step removes about that fraction of the residual, and an
 * inner solve far below it only adds iterations.  rtol outside (0, 1) only
 * reads the setting.  Process-wide; returns the previous setting.  No
 * counterpart in the reference. */
double asgk_set_bf16_inner_tol(double rtol);

/* ------------------------------------------------ implicit time loop */

typedef enum asgk_pc_kind
{
  ASGK_PC_NONE    = 0,
  ASGK_PC_JACOBI  = 1, /* precond is an asgk_jacobi * */
  ASGK_PC_LEARNED = 2  /* precond is an asgk_mlp * */
} asgk_pc_kind;

/* `steps` backward-Euler steps of the implicit time loop, the GMRES branch of
 * implicit_advance (src/time_advance.cpp:308-470) with x resident on the
 * device between steps: per step, x += dt * f_k (sources and boundary terms
 * at t + dt, as the reference adds them; f_k = forcing + k*forcing_stride,
 * forcing_stride 0 reuses one vector, forcing NULL adds nothing), then
 * (I - dt*K) x_new = x by simple_gmres_euler starting from the right-hand
 * side (the reference's initial guess), x_new overwriting x.  Solver
 * arguments as asgk_gmres_euler / asgk_gmres_euler_jacobi; info[k] receives
 * step k, including a solve that stopped short of the tolerance
 * (info[k].status, the loop goes on as the reference's does).  An error
 * return of a solve (invalid argument, CUDA, allocation) stops the loop and
 * is returned.  A device buffer of one vector is allocated for the call. */
int asgk_implicit_advance(asgk_plan *plan, double dt, double *x, int steps,
                          const double *forcing, int64_t forcing_stride,
                          int restart, int max_outer, double tol, int tol_mode,
                          int precision, int pc_kind, void *precond,
                          asgk_gmres_info *info, asgk_stream stream);

/* ------------------------------------------------ IMEX time loop */

/* Events of the IMEX hook: the points where the reference's imex_advance
 * updates PDE-specific state. */
typedef enum asgk_imex_event
{
  ASGK_IMEX_BEFORE_EXPLICIT = 0, /* f: the state the stage's explicit apply
                                    reads (f_0, then f_1): the reference's
                                    Poisson update */
  ASGK_IMEX_BEFORE_IMPLICIT = 1  /* f: the stage's explicit result (f_1s, then
                                    f_2s): the reference's moments and
                                    coefficient regeneration */
} asgk_imex_event;

/* Called by asgk_imex_advance at each event of each stage (stage 0, 1) of
 * each step.  f is a device vector of the plans' size, valid during the call
 * (work on `stream`, or synchronise it first).  The hook may change the
 * plans' coefficients (asgk_plan_update_values / asgk_plan_update_terms),
 * as generate_all_coefficients does in the reference; a Jacobi
 * preconditioner built earlier is then kept as it is (a preconditioner, not
 * the inverse of the updated operator).  Return 0 to go on; any other value
 * stops the loop and is returned by asgk_imex_advance. */
typedef int (*asgk_imex_hook)(void *ctx, int step, int stage, int event,
                              const double *f, asgk_stream stream);

/* `steps` steps of the reference's two-stage IMEX scheme (imex_advance,
 * src/time_advance.cpp:477-990) with x resident on the device:
 *   f_1s = f_0 + dt E f_0;           f_1 solves (I - dt I_op) f_1 = f_1s
 *   f_2s = (f_0 + f_1 + dt E f_1)/2; f_2 solves (I - dt/2 I_op) f_2 = f_2s
 * E = explicit_plan (applied in FP64), I_op = implicit_plan.  The stage-1
 * solve starts from f_1s, the stage-2 solve from f_1, as the reference does
 * without a previous refined solution.  implicit_plan null: no implicit
 * part (the reference without a collision operator): f_1 = f_1s and the
 * step ends with f_2s.  The solves take restart, max_outer, tol, tol_mode
 * and precision as asgk_gmres_euler; pc_stage1 / pc_stage2 (or null) are
 * Jacobi preconditioners of the implicit plan for dt and dt/2 (one of
 * another shape or step size: ASGK_ERR_INVALID before any work).  hook (or
 * null) with hook_ctx: see asgk_imex_hook.  info receives 2 entries per
 * step (stage 1, stage 2; zeros without an implicit plan), including
 * solves that stopped short of the tolerance (the loop goes on, as the
 * reference's does).  x is f_0 on entry and the last step's result on exit.
 * work: 4 vectors of the plans' size (device, contiguous: f_0, the explicit
 * product, f_1, the stage-1 solution), or null to have them allocated for
 * the call; every f a hook receives is x or one of them. */
int asgk_imex_advance(asgk_plan *explicit_plan, asgk_plan *implicit_plan,
                      double dt, double *x, int steps, int restart,
                      int max_outer, double tol, int tol_mode, int precision,
                      asgk_jacobi *pc_stage1, asgk_jacobi *pc_stage2,
                      asgk_imex_hook hook, void *hook_ctx, double *work,
                      asgk_gmres_info *info, asgk_stream stream);

/* ------------------------------------------------ learned preconditioner */

/* A per-cell learned preconditioner (no counterpart in the reference, which
 * has none on this path).  4 layers of width
 * `hidden` with GELU: the cell's residual block (scaled to unit norm) passes
 * through 4 linear layers whose hidden activations are gated elementwise by
 * GELU gates computed from the cell's level multi-index, so the network is
 * linear in the residual and the preconditioner
 *   z_c = ||v_c|| * f(v_c / ||v_c||, levels_c / max_level)
 * is a fixed linear operator, an approximation of (I - dt K)^{-1}.  FP32
 * master weights, BF16 tensor-core GEMMs with FP32 accumulation.
 * cell_levels: num_cells x d host ints (the element table's level columns).
 * Weights are initialised from seed. */
int asgk_mlp_create(asgk_mlp **mlp, int d, int n, int num_cells,
                    const int *cell_levels, int max_level, int hidden,
                    uint64_t seed);
void asgk_mlp_destroy(asgk_mlp *mlp);
int asgk_mlp_num_params(const asgk_mlp *mlp, int64_t *count);
/* Flat FP32 host layout: W1 (n^d x hidden), W2, W3 (hidden x hidden),
 * W4 (hidden x n^d), then per gated layer l = 1..3 the gate weights
 * (d x hidden) and gate biases (hidden); matrices row-major. */
int asgk_mlp_get_params(const asgk_mlp *mlp, float *params);
int asgk_mlp_set_params(asgk_mlp *mlp, const float *params);
/* One forward and backward pass on host rows (X: rows x (n^d + d), the
 * residual block then the level features; targets T: rows x n^d; FP32):
 * outputs Y, loss = 0.5*sum((Y - T)^2) and the gradients in the parameter
 * layout.  Used to check the kernels' gradients. */
int asgk_mlp_forward_backward(asgk_mlp *mlp, int rows, const float *X,
                              const float *T, float *Y, float *grads,
                              double *loss);
/* Trains on num_samples (v, e) vector pairs on the device (sample-major,
 * num_cells*n^d FP64 each, e = (I - dt K)^{-1} v): one row per (sample,
 * cell), mini-batches of `batch` rows, `epochs` passes, Adam(lr).  Reports
 * the last epoch's mean squared error.  Targets are e_c/||v_c||. */
int asgk_mlp_train(asgk_mlp *mlp, const double *v, const double *e,
                   int num_samples, int epochs, int batch, float lr,
                   uint64_t seed, double *final_loss, asgk_stream stream);
/* Residual-space training on the same (residual, GMRES-correction) pairs
 * (r_k, e_k), A e_k = r_k, A = I - dt K: minimises
 * ||A (M r_k - e_k)||^2 / ||r_k||^2 = ||A M r_k - r_k||^2 / ||r_k||^2 per
 * sample (one Adam step per sample, all cells in one batch).  plan_T holds
 * K^T on the same pair list (its gradient needs A^T); the operator applies
 * run in `precision`.  Reports the last epoch's mean loss. */
int asgk_mlp_train_residual(asgk_mlp *mlp, asgk_plan *plan, asgk_plan *plan_T,
                            double dt, const double *r, const double *e,
                            int num_samples, int epochs, float lr,
                            int precision, uint64_t seed, double *final_loss,
                            asgk_stream stream);
/* Makes the preconditioner base(v) + network(v): the network then learns a
 * correction to base (a Jacobi preconditioner, which must outlive this use;
 * NULL removes it).  The training entries are unchanged: pass them the
 * corrections e - base(r) as targets.  No counterpart in the reference. */
int asgk_mlp_set_base(asgk_mlp *mlp, asgk_jacobi *base);
/* z = M(v) on device vectors of the plan's size (base included). */
int asgk_mlp_apply(asgk_mlp *mlp, asgk_plan *plan, const double *v, double *z,
                   asgk_stream stream);

/* ------------------------------------------------------- sparse grids */

/* Host-side builder of the reference's sparse-grid operator structure:
 * element table (src/elements.cpp:248-351), 1D connectivity (connect_1d,
 * src/asgard_grid_1d.hpp) and connected cell pairs (check_connected,
 * src/asgard_kronmult_matrix.cpp:230-300).  Two-call: pass NULL arrays to get
 * the sizes. */
int64_t asgk_sparse_grid(int d, int level, int *table);
int asgk_connect_1d(int level, int *num_rows, int *num_conn, int *pntr,
                    int *indx);
int asgk_build_pairs(int d, int level, int num_cells, const int *table,
                     int64_t *nnz, int64_t *row_ptr, int *col_indx,
                     int *conn);
/* The pairs of the global form: per cell r, every cell c that agrees with r
 * in all dimensions but one (dim[i] = k, or c = r once per dimension) and
 * whose 1D cell in dimension k is connected to r's (conn[i] = that 1D
 * connection).  Two-call like asgk_build_pairs (NULL arrays: size only). */
int asgk_direction_pairs(int d, int level, int num_cells, const int *table,
                         int64_t *nnz, int64_t *row_ptr, int *col_indx,
                         int *dim, int *conn);

/* ------------------------------------------------------------ misc */

const char *asgk_status_string(int status);
/* Number of kernels this library launched since load (for launch counts). */
int64_t asgk_launch_count(void);
/* Measured FMA throughput (TFLOP/s, 2 flops per FMA) of the current device
 * for precision ASGK_FP64 or ASGK_FP32: the denominator of the roofline of the
 * CUDA-core kronmult kernels.  No counterpart in the reference. */
int asgk_measure_fma_peak(int precision, double *tflops);
/* Reads (and, if reset != 0, clears) the library's device-side error word:
 * ASGK_OK, or ASGK_ERR_DEVICE_TIMEOUT when a kernel gave up a bounded wait on
 * its shared-memory copies (it then skips its remaining work and returns,
 * so the GPU stays usable).  Synchronises the device.  No counterpart in the
 * reference, whose kernels have no waits. */
int asgk_device_status(int reset);
/* Device properties (SM count etc.) for the current device. */
int asgk_device_info(int *sm_count, int *cc_major, int *cc_minor);

#ifdef __cplusplus
}
#endif
#endif /* ASGARD_B200_H */
