/* Test infrastructure only: a plain-C restatement of the reference's CPU
 * algorithms on the kronmult + implicit GMRES path.  Used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker;
 * the product never links or calls it.
 *
 * Reference files cited per function in asgard_oracle.c.
 */
#ifndef ASGARD_ORACLE_H
#define ASGARD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = beta*y + alpha * sum_{pairs, terms} (A_0 (x) ... (x) A_{d-1}) x_col,
 * CSR pair format of kronmult::cpu_sparse. */
int orc_kronmult_sparse_f64(int d, int n, int rows, const int *pntr,
                            const int *indx, int terms, const int *iA,
                            const double *vA, double alpha, const double *x,
                            double beta, double *y);
int orc_kronmult_sparse_f32(int d, int n, int rows, const int *pntr,
                            const int *indx, int terms, const int *iA,
                            const float *vA, float alpha, const float *x,
                            float beta, float *y);

/* Dense form of kronmult::cpu_dense: every output cell r < rows with every
 * input cell c < cols; factor (t, k) of the pair is the n x n block of vA[t]
 * at k*nb^2*n^2 + (ic*nb + ir)*n^2, ir / ic the 1D indices of cells
 * r + row_offset / c + col_offset in elem (d ints per cell). */
int orc_kronmult_dense_f64(int d, int n, int rows, int cols, int terms,
                           const int *elem, int row_offset, int col_offset,
                           const double *const *vA, int nb, double alpha,
                           const double *x, double beta, double *y);
int orc_kronmult_dense_f32(int d, int n, int rows, int cols, int terms,
                           const int *elem, int row_offset, int col_offset,
                           const float *const *vA, int nb, float alpha,
                           const float *x, float beta, float *y);

/* Explicit Kronecker product of the d factors (pA[0] outermost) applied by a
 * dense GEMV: y += K x. */
void orc_reference_kronmult_one(int d, int n, const double *const *pA,
                                const double *x, double *y);

/* Dense assembly of the whole operator (N x N column-major, N = rows*n^d). */
int orc_assemble_dense(int d, int n, int rows, const int *pntr,
                       const int *indx, int terms, const int *iA,
                       const double *vA, double *K);

/* 1D hierarchical connectivity (connect_1d, full mode). Arrays nullable. */
int orc_connect_1d(int max_level, int *num_rows, int *num_conn, int *pntr,
                   int *indx);

/* Sparse grid: level multi-indexes with sum <= L, each expanded to cells, in
 * element-table order. table gets 2*d ints per cell. table nullable. */
int64_t orc_sparse_grid(int d, int L, int *table);

/* Connected cell pairs of a table (check_connected rule), CSR over rows, and
 * per pair the d 1D connection indices (offsets into connect_1d). Two-call:
 * with pntr/indx/conn null only *nnz is computed. */
int orc_build_pairs(int d, int L, int num_cells, const int *table,
                    int64_t *nnz, int *pntr, int *indx, int *conn);

/* Expands per-pair connection indices into reference iA offsets. */
void orc_expand_iA(int d, int n, int terms, int64_t nnz, const int *conn,
                   int *iA);

/* Reference BLAS Givens generation / application. */
void orc_rotg(double *a, double *b, double *c, double *s);

/* Restarted GMRES as in solver::simple_gmres, matrix-free over the sparse
 * kronmult for (I - dt K) x = b.  Absolute tolerance on the estimated
 * residual, classical Gram-Schmidt, Givens rotations, packed Hessenberg. */
int orc_gmres_euler(int d, int n, int rows, const int *pntr, const int *indx,
                    int terms, const int *iA, const double *vA, double dt,
                    double *x, const double *b, int restart, int max_outer,
                    double tol, double *err, int *iters);

/* Same GMRES over a dense column-major matrix (no preconditioner). */
int orc_gmres_dense(int n, const double *A, double *x, const double *b,
                    int restart, int max_outer, double tol, double *err,
                    int *iters);

/* std::minstd_rand + std::uniform_real_distribution (libstdc++ semantics). */
typedef struct { uint64_t state; } orc_minstd;
void orc_minstd_seed(orc_minstd *g, uint64_t seed);
double orc_uniform_f64(orc_minstd *g, double a, double b);
float orc_uniform_f32(orc_minstd *g, float a, float b);

/* make_kronmult_data(d, n, rows, terms, mats) with a sequential generator:
 * fills the CSR pair format (all rows x rows pairs), iA, vA, x, y0.
 * precision 8 = double, 4 = float (vA/x/y are of that type). */
int orc_make_kronmult_data(int d, int n, int rows, int terms, int mats,
                           int precision, int *pntr, int *indx, int *iA,
                           void *vA, void *x, void *y);

/* make_kronmult_welem(d, n, terms, range) of the dense tests: elem[range^d
 * * d], coeff[terms * d*range^2*n^2] (term-major), x and y [range^d * n^d]. */
int orc_make_kronmult_welem(int d, int n, int terms, int range, int precision,
                            int *elem, void *coeff, void *x, void *y);

#ifdef __cplusplus
}
#endif
#endif
