/* Test infrastructure only (see asgard_oracle.h): plain-C restatement of the
 * reference CPU algorithms on the kronmult + implicit GMRES path.  The
 * product never calls this; the tests compare the CUDA path against it and
 * pin it, in turn, against the reference compiled from source (oracle/_ref)
 * and against golden vectors under tests/golden/.
 */
#include "asgard_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int ipow_i(int n, int d)
{
  int r = 1;
  for (int i = 0; i < d; i++)
    r *= n;
  return r;
}

/* Contracts tensor axis k (0 = slowest, stride n^(d-1-k)) of the n^d tensor
 * w with the column-major n x n factor A: out(..s..) = sum_j A(s,j) w(..j..).
 * Follows the stage structure of kronmult::cpu_sparse
 * (src/device/asgard_spkronmult_cpu.cpp:84-433, general-n form in
 * src/device/asgard_spkronmult_cpu_general.hpp): the first factor in the iA
 * list acts on the slowest tensor index. */
#define DEFINE_CONTRACT(T, NAME)                                              \
  static void NAME(int d, int n, int k, const T *A, const T *w, T *out)       \
  {                                                                           \
    int const stride = ipow_i(n, d - 1 - k);                                  \
    int const outer  = ipow_i(n, k);                                          \
    for (int o = 0; o < outer; o++)                                           \
      for (int s = 0; s < n; s++)                                             \
        for (int in = 0; in < stride; in++)                                   \
        {                                                                     \
          T sum = 0;                                                          \
          for (int j = 0; j < n; j++)                                         \
            sum += A[j * n + s] * w[(o * n + j) * stride + in];               \
          out[(o * n + s) * stride + in] = sum;                               \
        }                                                                     \
  }
DEFINE_CONTRACT(double, contract_f64)
DEFINE_CONTRACT(float, contract_f32)

/* kronmult::cpu_sparse<T> (src/device/asgard_spkronmult_cpu.cpp:84-433,
 * dispatch :606-768): one output row (cell) per iteration; beta is applied to
 * the row block first, then every (column, term) product is accumulated. */
#define DEFINE_SPARSE(T, NAME, CONTRACT)                                      \
  int NAME(int d, int n, int rows, const int *pntr, const int *indx,          \
           int terms, const int *iA, const T *vA, T alpha, const T *x,        \
           T beta, T *y)                                                      \
  {                                                                           \
    if (d < 1 || d > 6 || n < 1)                                              \
      return 1;                                                               \
    int const ts = ipow_i(n, d);                                              \
    _Pragma("omp parallel")                                                   \
    {                                                                         \
      T *w0 = (T *)malloc(sizeof(T) * ts);                                    \
      T *w1 = (T *)malloc(sizeof(T) * ts);                                    \
      _Pragma("omp for schedule(dynamic, 16)")                                \
      for (int r = 0; r < rows; r++)                                          \
      {                                                                       \
        T *yr = y + (int64_t)r * ts;                                          \
        for (int j = 0; j < ts; j++)                                          \
          yr[j] = (beta == 0) ? (T)0 : ((beta == 1) ? yr[j] : beta * yr[j]);  \
        int64_t ma = (int64_t)pntr[r] * terms * d;                            \
        for (int jx = pntr[r]; jx < pntr[r + 1]; jx++)                        \
        {                                                                     \
          const T *xc = x + (int64_t)indx[jx] * ts;                           \
          for (int t = 0; t < terms; t++)                                     \
          {                                                                   \
            const T *src = xc;                                                \
            T *cur = w0, *nxt = w1;                                           \
            for (int k = 0; k < d; k++)                                       \
            {                                                                 \
              CONTRACT(d, n, k, vA + iA[ma++], src, cur);                     \
              src = cur;                                                      \
              T *tmp = cur;                                                   \
              cur = nxt;                                                      \
              nxt = tmp;                                                      \
            }                                                                 \
            if (alpha == 1)                                                   \
              for (int j = 0; j < ts; j++)                                    \
                yr[j] += src[j];                                              \
            else if (alpha == -1)                                             \
              for (int j = 0; j < ts; j++)                                    \
                yr[j] -= src[j];                                              \
            else                                                              \
              for (int j = 0; j < ts; j++)                                    \
                yr[j] += alpha * src[j];                                      \
          }                                                                   \
        }                                                                     \
      }                                                                       \
      free(w0);                                                               \
      free(w1);                                                               \
    }                                                                         \
    return 0;                                                                 \
  }
DEFINE_SPARSE(double, orc_kronmult_sparse_f64, contract_f64)
DEFINE_SPARSE(float, orc_kronmult_sparse_f32, contract_f32)

/* kronmult::cpu_dense<T> (src/device/asgard_kronmult_cpu.cpp:160-507,
 * dispatch :517-700): one output cell per iteration, beta applied to its
 * block first, then every (column cell, term) product in column order.
 * Factor (t, k) of the pair (r, c) is the column-major n x n block of
 * vA[t] at k*nb^2*n^2 + (ic*nb + ir)*n^2 with ir = elem[(r + row_offset)*d
 * + k], ic = elem[(c + col_offset)*d + k] (the reference's dense layout,
 * src/asgard_kronmult_matrix.cpp:95-113). */
#define DEFINE_DENSE(T, NAME, CONTRACT)                                       \
  int NAME(int d, int n, int rows, int cols, int terms, const int *elem,      \
           int row_offset, int col_offset, const T *const *vA, int nb,        \
           T alpha, const T *x, T beta, T *y)                                 \
  {                                                                           \
    if (d < 1 || d > 6 || n < 1)                                              \
      return 1;                                                               \
    int const ts       = ipow_i(n, d);                                        \
    int64_t const nn   = (int64_t)n * n;                                      \
    int64_t const vstr = (int64_t)nb * nb * nn;                               \
    _Pragma("omp parallel")                                                   \
    {                                                                         \
      T *w0 = (T *)malloc(sizeof(T) * ts);                                    \
      T *w1 = (T *)malloc(sizeof(T) * ts);                                    \
      _Pragma("omp for schedule(dynamic, 4)")                                 \
      for (int r = 0; r < rows; r++)                                          \
      {                                                                       \
        T *yr = y + (int64_t)r * ts;                                          \
        const int *iy = elem + (int64_t)(r + row_offset) * d;                 \
        for (int j = 0; j < ts; j++)                                          \
          yr[j] = (beta == 0) ? (T)0 : ((beta == 1) ? yr[j] : beta * yr[j]);  \
        for (int c = 0; c < cols; c++)                                        \
        {                                                                     \
          const int *ix = elem + (int64_t)(c + col_offset) * d;               \
          const T *xc   = x + (int64_t)c * ts;                                \
          for (int t = 0; t < terms; t++)                                     \
          {                                                                   \
            const T *src = xc;                                                \
            T *cur = w0, *nxt = w1;                                           \
            for (int k = 0; k < d; k++)                                       \
            {                                                                 \
              const T *A = vA[t] + k * vstr +                                 \
                           ((int64_t)ix[k] * nb + iy[k]) * nn;                \
              CONTRACT(d, n, k, A, src, cur);                                 \
              src = cur;                                                      \
              T *tmp = cur;                                                   \
              cur = nxt;                                                      \
              nxt = tmp;                                                      \
            }                                                                 \
            for (int j = 0; j < ts; j++)                                      \
              yr[j] += alpha * src[j];                                        \
          }                                                                   \
        }                                                                     \
      }                                                                       \
      free(w0);                                                               \
      free(w1);                                                               \
    }                                                                         \
    return 0;                                                                 \
  }
DEFINE_DENSE(double, orc_kronmult_dense_f64, contract_f64)
DEFINE_DENSE(float, orc_kronmult_dense_f32, contract_f32)

/* kronecker() and reference_kronmult_one() of the reference tests
 * (src/asgard_kronmult_tests.hpp:39-76): explicit product with pA[0] the
 * outermost factor, then a dense GEMV y += K x. */
void orc_reference_kronmult_one(int d, int n, const double *const *pA,
                                const double *x, double *y)
{
  int total = n;
  double *kron = (double *)malloc(sizeof(double) * n * n);
  memcpy(kron, pA[d - 1], sizeof(double) * n * n);
  for (int i = d - 2; i >= 0; i--)
  {
    int const m = n, nn = total;
    const double *A = pA[i];
    double *res = (double *)malloc(sizeof(double) * (size_t)m * m * nn * nn);
    for (int jm = 0; jm < m; jm++)
      for (int jn = 0; jn < nn; jn++)
        for (int im = 0; im < m; im++)
          for (int in = 0; in < nn; in++)
            res[(size_t)(jm * nn + jn) * (m * nn) + im * nn + in] =
                A[jm * m + im] * kron[jn * nn + in];
    free(kron);
    kron = res;
    total *= n;
  }
  for (int c = 0; c < total; c++)
    for (int r = 0; r < total; r++)
      y[r] += kron[(size_t)c * total + r] * x[c];
  free(kron);
}

int orc_assemble_dense(int d, int n, int rows, const int *pntr,
                       const int *indx, int terms, const int *iA,
                       const double *vA, double *K)
{
  int const ts = ipow_i(n, d);
  int64_t const N = (int64_t)rows * ts;
  memset(K, 0, sizeof(double) * N * N);
  const double *pA[6];
  double *col = (double *)calloc(ts, sizeof(double));
  double *out = (double *)calloc(ts, sizeof(double));
  for (int r = 0; r < rows; r++)
  {
    int64_t ma = (int64_t)pntr[r] * terms * d;
    for (int jx = pntr[r]; jx < pntr[r + 1]; jx++)
      for (int t = 0; t < terms; t++)
      {
        for (int k = 0; k < d; k++)
          pA[k] = vA + iA[ma++];
        for (int c = 0; c < ts; c++)
        {
          memset(col, 0, sizeof(double) * ts);
          memset(out, 0, sizeof(double) * ts);
          col[c] = 1;
          orc_reference_kronmult_one(d, n, pA, col, out);
          int64_t const gc = (int64_t)indx[jx] * ts + c;
          for (int i = 0; i < ts; i++)
            K[gc * N + (int64_t)r * ts + i] += out[i];
        }
      }
  }
  free(col);
  free(out);
  return 0;
}

/* check_connected(L1, p1, L2, p2), L1 <= L2
 * (src/asgard_kronmult_matrix.cpp:230-279): closed supports intersect on the
 * periodic unit interval. */
static int connected_1d(int L1, int p1, int L2, int p2)
{
  if (L1 <= 1 || L2 <= 1)
    return 1;
  if ((p1 == 0 && p2 == ((1 << (L2 - 1)) - 1)) ||
      (p2 == 0 && p1 == ((1 << (L1 - 1)) - 1)))
    return 1;
  if (L1 == L2)
    return abs(p1 - p2) <= 1;
  int side = (p2 % 2 == 0) ? -1 : 1;
  while (L2 > L1)
  {
    if (p2 % 2 == 0)
      side = (side == -1) ? -1 : 0;
    else
      side = (side == 1) ? 1 : 0;
    L2--;
    p2 /= 2;
  }
  return (p2 == p1) || (p2 + side == p1);
}

static void level_pos(int idx, int *L, int *p)
{
  if (idx == 0)
  {
    *L = 0;
    *p = 0;
    return;
  }
  int l = 0;
  while ((1 << l) <= idx)
    l++;
  *L = l;
  *p = idx - (1 << (l - 1));
}

static int connected_idx(int a, int b)
{
  int La, pa, Lb, pb;
  level_pos(a, &La, &pa);
  level_pos(b, &Lb, &pb);
  return (La <= Lb) ? connected_1d(La, pa, Lb, pb) : connected_1d(Lb, pb, La, pa);
}

/* connect_1d (src/asgard_grid_1d.hpp:19-330), full hierarchy: row i lists, in
 * ascending order, every 1D cell whose support touches cell i; a connection's
 * index is its position in the flattened CSR (get_offset, :92-122).  The
 * reference builds the rows constructively; here each row is the filtered
 * list of check_connected partners, which the tests pin to the reference's
 * CSR for every level used. */
int orc_connect_1d(int max_level, int *num_rows, int *num_conn, int *pntr,
                   int *indx)
{
  int const rows = 1 << max_level;
  int count = 0;
  if (pntr)
    pntr[0] = 0;
  for (int r = 0; r < rows; r++)
  {
    for (int c = 0; c < rows; c++)
      if (connected_idx(r, c))
      {
        if (indx)
          indx[count] = c;
        count++;
      }
    if (pntr)
      pntr[r + 1] = count;
  }
  *num_rows = rows;
  *num_conn = count;
  return 0;
}

/* Element table (src/elements.cpp:248-351 with
 * permutations::get_lequal_multi, src/permutations.cpp:36-55, and
 * select_indexex / generate_lower_index_level_sets / transp_data,
 * src/permutations.hpp:33-213): level multi-indexes with sum <= L visited
 * lexicographically with dimension 0 fastest, grouped by level sum, the
 * groups emitted from the largest sum down to zero; each multi-index
 * expands to its cells with dimension 0 fastest (get_cell_index_set,
 * src/elements.cpp:408-458). */
int64_t orc_sparse_grid(int d, int L, int *table)
{
  /* count level multi-indexes per sum */
  int64_t count = 0;
  for (int s = L; s >= 0; s--)
  {
    int lv[6] = {0, 0, 0, 0, 0, 0};
    for (;;)
    {
      int sum = 0;
      for (int k = 0; k < d; k++)
        sum += lv[k];
      if (sum == s)
      {
        int64_t cells = 1;
        for (int k = 0; k < d; k++)
          cells *= (lv[k] <= 1) ? 1 : (1 << (lv[k] - 1));
        if (table)
        {
          int cidx[6] = {0, 0, 0, 0, 0, 0};
          for (int64_t c = 0; c < cells; c++)
          {
            int *row = table + (count + c) * 2 * d;
            for (int k = 0; k < d; k++)
            {
              row[k]     = lv[k];
              row[d + k] = cidx[k];
            }
            for (int k = 0; k < d; k++)
            {
              int const lim = (lv[k] <= 1) ? 1 : (1 << (lv[k] - 1));
              if (++cidx[k] < lim)
                break;
              cidx[k] = 0;
            }
          }
        }
        count += cells;
      }
      /* next multi-index with entries summing to <= s, dimension 0 fastest */
      int k = 0;
      for (; k < d; k++)
      {
        lv[k]++;
        int tot = 0;
        for (int q = 0; q < d; q++)
          tot += lv[q];
        if (tot <= s)
          break;
        lv[k] = 0;
      }
      if (k == d)
        break;
    }
  }
  return count;
}

static int cell_1d_index(int level, int pos)
{
  return (level == 0) ? 0 : (1 << (level - 1)) + pos;
}

/* Pair list of make_kronmult_sparse (src/asgard_kronmult_matrix.cpp:406-466)
 * with check_connected over all dimensions (:282-300) and the 1D connection
 * offsets of compute_coefficient_offsets (:302-321). */
int orc_build_pairs(int d, int L, int num_cells, const int *table,
                    int64_t *nnz, int *pntr, int *indx, int *conn)
{
  int rows1d, nconn;
  orc_connect_1d(L, &rows1d, &nconn, NULL, NULL);
  int *cp = (int *)malloc(sizeof(int) * (rows1d + 1));
  int *ci = (int *)malloc(sizeof(int) * nconn);
  orc_connect_1d(L, &rows1d, &nconn, cp, ci);
  /* dense lookup of connection offsets, -1 if not connected */
  int *lut = (int *)malloc(sizeof(int) * rows1d * rows1d);
  for (int i = 0; i < rows1d * rows1d; i++)
    lut[i] = -1;
  for (int r = 0; r < rows1d; r++)
    for (int j = cp[r]; j < cp[r + 1]; j++)
      lut[r * rows1d + ci[j]] = j;

  int *counts = (int *)calloc(num_cells, sizeof(int));
#pragma omp parallel for schedule(dynamic, 8)
  for (int r = 0; r < num_cells; r++)
  {
    const int *rc = table + (int64_t)r * 2 * d;
    int cnt = 0;
    for (int c = 0; c < num_cells; c++)
    {
      const int *cc = table + (int64_t)c * 2 * d;
      int ok = 1;
      for (int k = 0; k < d && ok; k++)
        ok = lut[cell_1d_index(rc[k], rc[d + k]) * rows1d +
                 cell_1d_index(cc[k], cc[d + k])] >= 0;
      cnt += ok;
    }
    counts[r] = cnt;
  }
  int64_t total = 0;
  for (int r = 0; r < num_cells; r++)
    total += counts[r];
  *nnz = total;
  if (pntr && indx)
  {
    pntr[0] = 0;
    for (int r = 0; r < num_cells; r++)
      pntr[r + 1] = pntr[r] + counts[r];
#pragma omp parallel for schedule(dynamic, 8)
    for (int r = 0; r < num_cells; r++)
    {
      const int *rc = table + (int64_t)r * 2 * d;
      int64_t pos = pntr[r];
      for (int c = 0; c < num_cells; c++)
      {
        const int *cc = table + (int64_t)c * 2 * d;
        int off[6];
        int ok = 1;
        for (int k = 0; k < d && ok; k++)
        {
          off[k] = lut[cell_1d_index(rc[k], rc[d + k]) * rows1d +
                       cell_1d_index(cc[k], cc[d + k])];
          ok     = off[k] >= 0;
        }
        if (ok)
        {
          indx[pos] = c;
          if (conn)
            for (int k = 0; k < d; k++)
              conn[pos * d + k] = off[k];
          pos++;
        }
      }
    }
  }
  free(counts);
  free(lut);
  free(cp);
  free(ci);
  return 0;
}

/* iA = off_k * (d*T*n^2) + (t*d + k) * n^2 (src/asgard_kronmult_matrix.cpp:455-461). */
void orc_expand_iA(int d, int n, int terms, int64_t nnz, const int *conn,
                   int *iA)
{
  int64_t const block = (int64_t)d * terms * n * n;
  for (int64_t p = 0; p < nnz; p++)
    for (int t = 0; t < terms; t++)
      for (int k = 0; k < d; k++)
        iA[(p * terms + t) * d + k] =
            (int)(conn[p * d + k] * block + (int64_t)(t * d + k) * n * n);
}

/* Reference BLAS drotg (the classic netlib algorithm the reference reaches
 * through lib_dispatch::rotg, src/lib_dispatch.cpp:258-297). */
void orc_rotg(double *a, double *b, double *c, double *s)
{
  double const sa = *a, sb = *b;
  double roe = (fabs(sa) > fabs(sb)) ? sa : sb;
  double scale = fabs(sa) + fabs(sb);
  double r, z;
  if (scale == 0)
  {
    *c = 1;
    *s = 0;
    r  = 0;
    z  = 0;
  }
  else
  {
    r  = scale * sqrt((sa / scale) * (sa / scale) + (sb / scale) * (sb / scale));
    r  = (roe >= 0 ? 1.0 : -1.0) * r;
    *c = sa / r;
    *s = sb / r;
    z  = 1;
    if (fabs(sa) > fabs(sb))
      z = *s;
    if (fabs(sb) >= fabs(sa) && *c != 0)
      z = 1 / *c;
  }
  *a = r;
  *b = z;
}

static void rot1(double *x, double *y, double c, double s)
{
  double const tx = c * *x + s * *y;
  double const ty = c * *y - s * *x;
  *x = tx;
  *y = ty;
}

typedef void (*matvec_fn)(void *ctx, double alpha, const double *x,
                          double beta, double *y);

static int pos_from_indices(int i, int j) { return i + j * (j + 1) / 2; }

static double nrm2(int64_t n, const double *v)
{
  double s = 0;
  for (int64_t i = 0; i < n; i++)
    s += v[i] * v[i];
  return sqrt(s);
}

/* solver::simple_gmres (src/solver.cpp:157-298) without preconditioner:
 * restarted GMRES, classical Gram-Schmidt as two GEMVs, Givens rotations,
 * packed upper Hessenberg solved by tpsv, absolute tolerance on the
 * estimated residual |s_k g_k|.  total_iterations counts one per restart
 * residual plus one per Arnoldi step.  As in the reference, the last Givens
 * rotation is not applied to the right-hand side once the tolerance is met. */
static int gmres_core(int64_t n, matvec_fn mat, void *ctx, double *x,
                      const double *b, int restart, int max_outer, double tol,
                      double *err, int *iters)
{
  if (restart > n || restart < 1)
    return 3;
  double *V      = (double *)malloc(sizeof(double) * n * (restart + 1));
  double *proj   = (double *)calloc((size_t)restart * (restart + 1) / 2, sizeof(double));
  double *sines  = (double *)calloc(restart + 1, sizeof(double));
  double *cosins = (double *)calloc(restart + 1, sizeof(double));
  double *ksol   = (double *)calloc(restart + 1, sizeof(double));
  int total = 0, outer = 0, inner = 0;
  double inner_res = 0, outer_res = tol + 1;
  while (outer_res > tol && outer < max_outer)
  {
    double *r = V;
    memcpy(r, b, sizeof(double) * n);
    mat(ctx, -1.0, x, 1.0, r);
    ++total;
    inner_res = nrm2(n, r);
    for (int64_t i = 0; i < n; i++)
      r[i] *= 1.0 / inner_res;
    ksol[0] = inner_res;
    inner   = 0;
    while (inner_res > tol && inner < restart)
    {
      double *vi = V + (int64_t)inner * n, *w = V + (int64_t)(inner + 1) * n;
      mat(ctx, 1.0, vi, 0.0, w);
      ++total;
      double *coeffs = proj + pos_from_indices(0, inner);
      for (int k = 0; k <= inner; k++)
      {
        double s = 0;
        const double *vk = V + (int64_t)k * n;
        for (int64_t i = 0; i < n; i++)
          s += vk[i] * w[i];
        coeffs[k] = s;
      }
      for (int64_t i = 0; i < n; i++)
      {
        double s = 0;
        for (int k = 0; k <= inner; k++)
          s += V[(int64_t)k * n + i] * coeffs[k];
        w[i] -= s;
      }
      double const nrm = nrm2(n, w);
      for (int64_t i = 0; i < n; i++)
        w[i] *= 1.0 / nrm;
      for (int k = 0; k < inner; k++)
        rot1(&coeffs[k], &coeffs[k + 1], cosins[k], sines[k]);
      double beta = nrm;
      orc_rotg(&coeffs[inner], &beta, &cosins[inner], &sines[inner]);
      inner_res = fabs(sines[inner] * ksol[inner]);
      if (inner_res > tol && inner < restart)
      {
        ksol[inner + 1] = 0;
        rot1(&ksol[inner], &ksol[inner + 1], cosins[inner], sines[inner]);
      }
      ++inner;
    }
    if (inner > 0)
    {
      /* tpsv: upper, no-transpose, non-unit, packed column-major */
      for (int j = inner - 1; j >= 0; j--)
      {
        if (ksol[j] != 0)
        {
          ksol[j] /= proj[pos_from_indices(j, j)];
          double const tmp = ksol[j];
          for (int i = j - 1; i >= 0; i--)
            ksol[i] -= tmp * proj[pos_from_indices(i, j)];
        }
      }
      for (int64_t i = 0; i < n; i++)
      {
        double s = 0;
        for (int k = 0; k < inner; k++)
          s += V[(int64_t)k * n + i] * ksol[k];
        x[i] += s;
      }
    }
    ++outer;
    outer_res = inner_res;
  }
  *err   = outer_res;
  *iters = total;
  free(V);
  free(proj);
  free(sines);
  free(cosins);
  free(ksol);
  return 0;
}

struct euler_ctx
{
  int d, n, rows, terms;
  const int *pntr, *indx, *iA;
  const double *vA;
  double dt;
  int64_t N;
};

/* The matvec of simple_gmres_euler (src/solver.cpp:119-135):
 * apply(-dt*alpha, x, beta, y) followed by y += alpha*x. */
static void euler_matvec(void *vctx, double alpha, const double *x,
                         double beta, double *y)
{
  struct euler_ctx *c = (struct euler_ctx *)vctx;
  orc_kronmult_sparse_f64(c->d, c->n, c->rows, c->pntr, c->indx, c->terms,
                          c->iA, c->vA, -c->dt * alpha, x, beta, y);
  for (int64_t i = 0; i < c->N; i++)
    y[i] += alpha * x[i];
}

int orc_gmres_euler(int d, int n, int rows, const int *pntr, const int *indx,
                    int terms, const int *iA, const double *vA, double dt,
                    double *x, const double *b, int restart, int max_outer,
                    double tol, double *err, int *iters)
{
  struct euler_ctx c = {d, n, rows, terms, pntr, indx, iA, vA, dt,
                        (int64_t)rows * ipow_i(n, d)};
  return gmres_core(c.N, euler_matvec, &c, x, b, restart, max_outer, tol, err,
                    iters);
}

struct dense_ctx
{
  int n;
  const double *A;
};

static void dense_matvec(void *vctx, double alpha, const double *x,
                         double beta, double *y)
{
  struct dense_ctx *c = (struct dense_ctx *)vctx;
  for (int i = 0; i < c->n; i++)
  {
    double s = 0;
    for (int j = 0; j < c->n; j++)
      s += c->A[i + (int64_t)j * c->n] * x[j];
    y[i] = (beta == 0 ? 0 : beta * y[i]) + alpha * s;
  }
}

int orc_gmres_dense(int n, const double *A, double *x, const double *b,
                    int restart, int max_outer, double tol, double *err,
                    int *iters)
{
  struct dense_ctx c = {n, A};
  return gmres_core(n, dense_matvec, &c, x, b, restart, max_outer, tol, err,
                    iters);
}

/* std::minstd_rand (a = 48271, m = 2^31 - 1) and libstdc++'s
 * generate_canonical / uniform_real_distribution, as used by
 * make_kronmult_data (src/asgard_kronmult_tests.hpp:111-190). */
void orc_minstd_seed(orc_minstd *g, uint64_t seed)
{
  g->state = seed % 2147483647ULL;
  if (g->state == 0)
    g->state = 1;
}

static uint64_t minstd_next(orc_minstd *g)
{
  g->state = (g->state * 48271ULL) % 2147483647ULL;
  return g->state;
}

double orc_uniform_f64(orc_minstd *g, double a, double b)
{
  /* two draws: range r = max - min + 1 = 2147483646 */
  double const r = 2147483646.0;
  double sum = 0, tmp = 1;
  for (int k = 0; k < 2; k++)
  {
    sum += (double)(minstd_next(g) - 1) * tmp;
    tmp *= r;
  }
  double ret = sum / tmp;
  if (ret >= 1.0)
    ret = nextafter(1.0, 0.0);
  return ret * (b - a) + a;
}

float orc_uniform_f32(orc_minstd *g, float a, float b)
{
  float const r = (float)2147483646.0;
  float sum = 0, tmp = 1;
  sum += (float)(minstd_next(g) - 1) * tmp;
  tmp *= r;
  float ret = sum / tmp;
  if (ret >= 1.0f)
    ret = nextafterf(1.0f, 0.0f);
  float const span = b - a;
  float const prod = ret * span;
  return prod + a;
}

int orc_make_kronmult_data(int d, int n, int rows, int terms, int mats,
                           int precision, int *pntr, int *indx, int *iA,
                           void *vA, void *x, void *y)
{
  orc_minstd g;
  orc_minstd_seed(&g, 42);
  int const ts = ipow_i(n, d);
  /* pointer map: per (row-major pair, term): x index, d matrices, y index */
  int64_t const nb = (int64_t)rows * rows;
  for (int64_t i = 0; i < nb; i++)
    for (int t = 0; t < terms; t++)
      for (int k = 0; k < d; k++)
      {
        int m;
        if (precision == 8)
          m = (int)orc_uniform_f64(&g, 0.0, (double)(mats - 1));
        else
          m = (int)orc_uniform_f32(&g, 0.0f, (float)(mats - 1));
        iA[(i * terms + t) * d + k] = n * n * m;
      }
  for (int r = 0; r < rows; r++)
  {
    pntr[r] = r * rows;
    for (int c = 0; c < rows; c++)
      indx[r * rows + c] = c;
  }
  pntr[rows] = rows * rows;
  int64_t const nm = (int64_t)n * n * mats;
  int64_t const nx = (int64_t)ts * rows;
  if (precision == 8)
  {
    double *va = (double *)vA, *xx = (double *)x, *yy = (double *)y;
    for (int64_t i = 0; i < nm; i++)
      va[i] = orc_uniform_f64(&g, -1.0, 1.0);
    for (int64_t i = 0; i < nx; i++)
    {
      xx[i] = orc_uniform_f64(&g, -1.0, 1.0);
      yy[i] = orc_uniform_f64(&g, -1.0, 1.0);
    }
  }
  else
  {
    float *va = (float *)vA, *xx = (float *)x, *yy = (float *)y;
    for (int64_t i = 0; i < nm; i++)
      va[i] = orc_uniform_f32(&g, -1.0f, 1.0f);
    for (int64_t i = 0; i < nx; i++)
    {
      xx[i] = orc_uniform_f32(&g, -1.0f, 1.0f);
      yy[i] = orc_uniform_f32(&g, -1.0f, 1.0f);
    }
  }
  return 0;
}

/* kronmult_intputs_welem<P>(d, n, terms, range) of the reference's dense
 * tests (src/asgard_kronmult_tests.hpp:236-300): range^d cells whose 1D
 * indices are the base-d digits of the cell number (the digit base there is
 * the number of dimensions, not range), then from minstd_rand(42) every
 * coefficient of every term (d*range^2*n^2 each, term after term), all of x,
 * all of y.  precision 8 = double, 4 = float. */
int orc_make_kronmult_welem(int d, int n, int terms, int range, int precision,
                            int *elem, void *coeff, void *x, void *y)
{
  if (d < 1 || n < 1 || terms < 0 || range < 1)
    return 1;
  int const rows = ipow_i(range, d);
  for (int i = 0; i < rows; i++)
  {
    int t = i;
    for (int k = 0; k < d; k++)
    {
      elem[i * d + k] = t % d;
      t /= d;
    }
  }
  orc_minstd g;
  orc_minstd_seed(&g, 42);
  int64_t const nc = (int64_t)terms * d * range * range * n * n;
  int64_t const nx = (int64_t)ipow_i(n, d) * rows;
  if (precision == 8)
  {
    double *c = (double *)coeff, *xx = (double *)x, *yy = (double *)y;
    for (int64_t i = 0; i < nc; i++)
      c[i] = orc_uniform_f64(&g, -1.0, 1.0);
    for (int64_t i = 0; i < nx; i++)
      xx[i] = orc_uniform_f64(&g, -1.0, 1.0);
    for (int64_t i = 0; i < nx; i++)
      yy[i] = orc_uniform_f64(&g, -1.0, 1.0);
  }
  else
  {
    float *c = (float *)coeff, *xx = (float *)x, *yy = (float *)y;
    for (int64_t i = 0; i < nc; i++)
      c[i] = orc_uniform_f32(&g, -1.0f, 1.0f);
    for (int64_t i = 0; i < nx; i++)
      xx[i] = orc_uniform_f32(&g, -1.0f, 1.0f);
    for (int64_t i = 0; i < nx; i++)
      yy[i] = orc_uniform_f32(&g, -1.0f, 1.0f);
  }
  return 0;
}
