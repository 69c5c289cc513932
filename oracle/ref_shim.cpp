// Test infrastructure: a C entry layer over the reference ASGarD library,
// compiled from the reference's own sources by oracle/Makefile into
// oracle/_ref/libasgard_ref.so.  Nothing in the product links this file; the
// tests, smoke() and the bench's CPU-baseline leg load it through ctypes as
// the checker and as the "reference" CPU timing arm.
//
// Everything here forwards to the reference code unchanged:
//   * kronmult::cpu_sparse               src/device/asgard_spkronmult_cpu.cpp:606-768
//   * kronmult_matrix<P> (CPU, sparse)   src/asgard_kronmult_matrix.hpp:235-297, 340-478
//   * kronmult_matrix<P> (CPU, dense)    src/asgard_kronmult_matrix.hpp:132-176 (cpu_dense)
//   * solver::simple_gmres_euler         src/solver.cpp:119-135
//   * solver::simple_gmres (dense)       src/solver.cpp:55-74
//   * connect_1d                         src/asgard_grid_1d.hpp:19-330
//   * make_kronmult_matrix (sparse)      src/asgard_kronmult_matrix.cpp:330-690
//   * compute_mem_usage                  src/asgard_kronmult_matrix.cpp:813-1004

// Pull in every standard header the reference uses before re-defining the
// access specifier below, so that only the reference's own classes are
// affected (the pair list built by make_kronmult_sparse is stored in private
// members and there is no accessor for it).
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <optional>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <variant>
#include <vector>
#include <omp.h>

#define private public
#define protected public
#include "asgard_kronmult_matrix.hpp"
#include "basis.hpp"
#include "coefficients.hpp"
#include "solver.hpp"
#include "asgard_kronmult_tests.hpp"
#undef private
#undef protected

using namespace asgard;

namespace
{
// Silences the reference's per-iteration std::cout prints while a call runs.
struct quiet_cout
{
  std::streambuf *old;
  std::ostringstream sink;
  explicit quiet_cout(bool on) : old(nullptr)
  {
    if (on)
      old = std::cout.rdbuf(sink.rdbuf());
  }
  ~quiet_cout()
  {
    if (old)
      std::cout.rdbuf(old);
  }
};

template<typename T>
kronmult_matrix<T>
make_cpu_sparse(int d, int n, int rows, int cols, int terms, int const *pntr,
                int const *indx, int const *iA, T const *vA, int64_t vA_len)
{
  int64_t const nnz = pntr[rows];
  std::vector<fk::vector<int>> lp, li, la;
  lp.push_back(fk::vector<int>(std::vector<int>(pntr, pntr + rows + 1)));
  li.push_back(fk::vector<int>(std::vector<int>(indx, indx + nnz)));
  la.push_back(fk::vector<int>(
      std::vector<int>(iA, iA + nnz * int64_t(d) * int64_t(terms))));
  fk::vector<T> va(std::vector<T>(vA, vA + vA_len));
  return kronmult_matrix<T>(d, n, rows, cols, terms, std::move(lp),
                            std::move(li), std::move(la), std::move(va));
}
// make_kronmult_data<T>(d, n, rows, terms, mats) of the reference tests
// (src/asgard_kronmult_tests.hpp:111-190), run on one OpenMP thread so the
// shared random engine is drawn in order, converted to the CSR pair format
// exactly as test_kronmult_sparse does (src/asgard_kronmult_matrix_tests.cpp:
// 14-118).  ref_y is the reference's explicit Kronecker-product answer for
// y <- y + K x (alpha = beta = 1).
template<typename T>
int make_data(int d, int n, int rows, int terms, int mats, int *pntr,
                     int *indx, int *iA, T *vA, T *x, T *y, T *ref_y)
{
  int const saved = omp_get_max_threads();
  omp_set_num_threads(1);
  auto data = make_kronmult_data<T, true>(d, n, rows, terms, mats);
  omp_set_num_threads(saved);
  int const num_batch = rows * rows;
  auto ip = data->pointer_map.begin();
  for (int i = 0; i < num_batch * terms; i++)
  {
    ip++;
    for (int j = 0; j < d; j++)
      iA[i * d + j] = n * n * (*ip++);
    ip++;
  }
  for (int i = 0; i < rows; i++)
  {
    pntr[i] = i * rows;
    for (int j = 0; j < rows; j++)
      indx[i * rows + j] = j;
  }
  pntr[rows] = num_batch;
  std::copy(data->matrices.begin(), data->matrices.end(), vA);
  std::copy(data->input_x.begin(), data->input_x.end(), x);
  std::copy(data->output_y.begin(), data->output_y.end(), y);
  std::copy(data->reference_y.begin(), data->reference_y.end(), ref_y);
  return 0;
}

// make_kronmult_welem<T>(d, n, terms, range) of the reference's dense tests
// (src/asgard_kronmult_tests.hpp:236-353): elem, the term coefficients
// (concatenated), x, y, and -- with want_ref -- its explicit
// Kronecker-product answer of y <- y + K x.
template<typename T>
int make_welem(int d, int n, int terms, int range, int want_ref, int *elem,
               T *coeff, T *x, T *y, T *ref_y)
{
  std::unique_ptr<kronmult_intputs_welem<T>> data;
  if (want_ref)
    data = make_kronmult_welem<T, true>(d, n, terms, range);
  else
    data = make_kronmult_welem<T, false>(d, n, terms, range);
  std::copy(data->elem.begin(), data->elem.end(), elem);
  for (auto const &c : data->coefficients)
    coeff = std::copy_n(c.data(), c.size(), coeff);
  std::copy(data->input_x.begin(), data->input_x.end(), x);
  std::copy(data->output_y.begin(), data->output_y.end(), y);
  std::copy(data->reference_y.begin(), data->reference_y.end(), ref_y);
  return 0;
}

// kronmult_matrix<T> through its dense constructor
// (src/asgard_kronmult_matrix.hpp:132-176) and apply (cpu_dense).
template<typename T>
int dense_apply(int d, int n, int rows, int cols, int terms, T const *coeff,
                int const *elem, int elem_len, int row_offset, int col_offset,
                int nb, T alpha, T const *x, T beta, T *y)
{
  try
  {
    int64_t const per = int64_t(d) * nb * nb * n * n;
    std::vector<fk::vector<T>> tv;
    for (int t = 0; t < terms; t++)
      tv.push_back(fk::vector<T>(std::vector<T>(coeff + t * per, coeff + (t + 1) * per)));
    fk::vector<int> el(std::vector<int>(elem, elem + elem_len));
    kronmult_matrix<T> mat(d, n, rows, cols, terms, std::move(tv), std::move(el),
                           row_offset, col_offset, nb);
    mat.apply(alpha, x, beta, y);
  }
  catch (std::exception const &)
  {
    return 1;
  }
  return 0;
}

} // namespace

extern "C"
{
int ref_num_threads() { return omp_get_max_threads(); }

// y = beta*y + alpha*K*x through kronmult::cpu_sparse (CSR pair format).
int ref_cpu_sparse_f64(int d, int n, int rows, int const *pntr,
                       int const *indx, int terms, int const *iA,
                       double const *vA, double alpha, double const *x,
                       double beta, double *y)
{
  try
  {
    kronmult::cpu_sparse<double>(d, n, rows, pntr, indx, terms, iA, vA, alpha,
                                 x, beta, y);
  }
  catch (std::exception const &)
  {
    return 1;
  }
  return 0;
}

int ref_cpu_sparse_f32(int d, int n, int rows, int const *pntr,
                       int const *indx, int terms, int const *iA,
                       float const *vA, float alpha, float const *x,
                       float beta, float *y)
{
  try
  {
    kronmult::cpu_sparse<float>(d, n, rows, pntr, indx, terms, iA, vA, alpha,
                                x, beta, y);
  }
  catch (std::exception const &)
  {
    return 1;
  }
  return 0;
}

// kronmult_matrix<double>::apply through the CPU sparse constructor.
int ref_kronmult_matrix_apply_f64(int d, int n, int rows, int cols, int terms,
                                  int const *pntr, int const *indx,
                                  int const *iA, double const *vA,
                                  int64_t vA_len, double alpha,
                                  double const *x, double beta, double *y)
{
  try
  {
    auto mat = make_cpu_sparse<double>(d, n, rows, cols, terms, pntr, indx, iA,
                                       vA, vA_len);
    mat.apply(alpha, x, beta, y);
  }
  catch (std::exception const &)
  {
    return 1;
  }
  return 0;
}

// solver::simple_gmres_euler on host vectors: solves (I - dt*K) x = b.
int ref_gmres_euler_f64(int d, int n, int rows, int terms, int const *pntr,
                        int const *indx, int const *iA, double const *vA,
                        int64_t vA_len, double dt, double *x, double const *b,
                        int restart, int max_iter, double tol, int quiet,
                        double *err, int *iters)
{
  try
  {
    auto mat = make_cpu_sparse<double>(d, n, rows, rows, terms, pntr, indx, iA,
                                       vA, vA_len);
    int64_t const N = int64_t(rows) * mat.tensor_size();
    fk::vector<double> fx(std::vector<double>(x, x + N));
    fk::vector<double> fb(std::vector<double>(b, b + N));
    quiet_cout q(quiet != 0);
    auto info = solver::simple_gmres_euler<double, resource::host>(
        dt, mat, fx, fb, restart, max_iter, tol);
    std::copy_n(fx.data(), N, x);
    *err   = info.error;
    *iters = info.iterations;
  }
  catch (std::exception const &)
  {
    return 1;
  }
  return 0;
}

// solver::simple_gmres on a dense column-major A, optional dense preconditioner M.
int ref_gmres_dense_f64(int n, double const *A, double *x, double const *b,
                        double const *M, int restart, int max_iter, double tol,
                        int quiet, double *err, int *iters)
{
  try
  {
    fk::matrix<double> fa(n, n);
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++)
        fa(i, j) = A[i + j * n];
    fk::matrix<double> fm;
    if (M != nullptr)
    {
      fm = fk::matrix<double>(n, n);
      for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++)
          fm(i, j) = M[i + j * n];
    }
    fk::vector<double> fx(std::vector<double>(x, x + n));
    fk::vector<double> fb(std::vector<double>(b, b + n));
    quiet_cout q(quiet != 0);
    auto info = solver::simple_gmres(fa, fx, fb, fm, restart, max_iter, tol);
    std::copy_n(fx.data(), n, x);
    *err   = info.error;
    *iters = info.iterations;
  }
  catch (std::exception const &)
  {
    return 1;
  }
  return 0;
}

// connect_1d(max_level, full): CSR of connected 1D hierarchical cells.
// Call once with null arrays to get the sizes.
int ref_connect_1d(int max_level, int *num_rows, int *num_conn, int *pntr,
                   int *indx, int *diag)
{
  connect_1d c(max_level);
  *num_rows = c.num_rows();
  *num_conn = c.num_connections();
  if (pntr)
    for (int r = 0; r <= c.num_rows(); r++)
      pntr[r] = (r < c.num_rows()) ? c.row_begin(r) : c.num_connections();
  if (indx)
    for (int j = 0; j < c.num_connections(); j++)
      indx[j] = c[j];
  if (diag)
    for (int r = 0; r < c.num_rows(); r++)
      diag[r] = c.row_diag(r);
  return 0;
}

int ref_connect_1d_offset(int max_level, int row, int col)
{
  connect_1d c(max_level);
  return c.get_offset(row, col);
}

// A built-in reference PDE discretised at (level, degree), with its sparse
// kronmult matrix made by the reference's own builder (CPU one-call format).
struct ref_pde
{
  std::unique_ptr<PDE<double>> pde;
  std::unique_ptr<options> opts;
  std::unique_ptr<adapt::distributed_grid<double>> grid;
  kron_sparse_cache spcache;
  memory_usage mem;
  kronmult_matrix<double> mat;
};

void *ref_pde_create(char const *name, char const *levels, int degree)
{
  try
  {
    quiet_cout q(true);
    std::vector<std::string> args = {"-p",           name,
                                     "-l",           levels,
                                     "-d",           std::to_string(degree),
                                     "--kron-mode",  "sparse",
                                     "-i",           "-s",
                                     "gmres"};
    std::vector<char const *> cargs = {"asgard"};
    for (auto &a : args)
      cargs.push_back(a.c_str());
    parser const cli(static_cast<int>(cargs.size()), cargs.data());
    auto h  = std::make_unique<ref_pde>();
    h->pde  = make_PDE<double>(cli);
    h->opts = std::make_unique<options>(cli);
    basis::wavelet_transform<double, resource::host> const transformer(
        *h->opts, *h->pde);
    generate_all_coefficients(*h->pde, transformer);
    h->grid = std::make_unique<adapt::distributed_grid<double>>(*h->pde,
                                                                 *h->opts);
    h->mem = compute_mem_usage(*h->pde, *h->grid, *h->opts,
                               imex_flag::unspecified, h->spcache, 0,
                               2147483646, true);
    h->mat = make_kronmult_matrix(*h->pde, *h->grid, *h->opts, h->mem,
                                  imex_flag::unspecified, h->spcache, true);
    return h.release();
  }
  catch (std::exception const &e)
  {
    std::cerr << "ref_pde_create: " << e.what() << "\n";
    return nullptr;
  }
}

void ref_pde_destroy(void *h) { delete static_cast<ref_pde *>(h); }

// sizes: d, n, rows, terms, max_level, nnz, iA length, vA length, dt
int ref_pde_info(void *hv, int *d, int *n, int *rows, int *terms,
                 int *max_level, int64_t *nnz, int64_t *iA_len,
                 int64_t *vA_len, double *dt)
{
  auto *h = static_cast<ref_pde *>(hv);
  auto &m = h->mat;
  if (m.list_row_indx_.size() != 1)
    return 2; // multi-call split: not exported
  *d         = m.num_dimensions_;
  *n         = m.kron_size_;
  *rows      = m.num_rows_;
  *terms     = m.num_terms_;
  *max_level = h->pde->max_level;
  *nnz       = m.list_col_indx_[0].size();
  *iA_len    = m.list_iA[0].size();
  *vA_len    = m.vA.size();
  *dt        = h->pde->get_dt();
  return 0;
}

// Exports the pair list (CSR), factor offsets, factor values and the
// element table (2*d ints per cell: levels then cell indices).
int ref_pde_export(void *hv, int *pntr, int *indx, int *iA, double *vA,
                   int *table)
{
  auto *h = static_cast<ref_pde *>(hv);
  auto &m = h->mat;
  std::copy_n(m.list_row_indx_[0].data(), m.list_row_indx_[0].size(), pntr);
  std::copy_n(m.list_col_indx_[0].data(), m.list_col_indx_[0].size(), indx);
  std::copy_n(m.list_iA[0].data(), m.list_iA[0].size(), iA);
  std::copy_n(m.vA.data(), m.vA.size(), vA);
  auto const &t = h->grid->get_table().get_active_table();
  std::copy_n(t.data(), t.size(), table);
  return 0;
}

// The full 1D operator matrix of (term, dim): (n 2^L) x (n 2^L), column-major.
int ref_pde_coefficients(void *hv, int term, int dim, double *out, int *lda)
{
  auto *h        = static_cast<ref_pde *>(hv);
  auto const &cm = h->pde->get_coefficients(term, dim);
  *lda           = cm.nrows();
  if (out)
    for (int j = 0; j < cm.ncols(); j++)
      for (int i = 0; i < cm.nrows(); i++)
        out[i + int64_t(j) * cm.nrows()] = cm(i, j);
  return 0;
}

int ref_pde_apply(void *hv, double alpha, double const *x, double beta,
                  double *y)
{
  auto *h = static_cast<ref_pde *>(hv);
  h->mat.apply(alpha, x, beta, y);
  return 0;
}

int ref_pde_gmres_euler(void *hv, double dt, double *x, double const *b,
                        int restart, int max_iter, double tol, int quiet,
                        double *err, int *iters)
{
  auto *h = static_cast<ref_pde *>(hv);
  int64_t const N = h->mat.output_size();
  fk::vector<double> fx(std::vector<double>(x, x + N));
  fk::vector<double> fb(std::vector<double>(b, b + N));
  quiet_cout q(quiet != 0);
  auto info = solver::simple_gmres_euler<double, resource::host>(
      dt, h->mat, fx, fb, restart, max_iter, tol);
  std::copy_n(fx.data(), N, x);
  *err   = info.error;
  *iters = info.iterations;
  return 0;
}

int ref_make_kronmult_data_f64(int d, int n, int rows, int terms, int mats,
                               int *pntr, int *indx, int *iA, double *vA,
                               double *x, double *y, double *ref_y)
{
  return make_data<double>(d, n, rows, terms, mats, pntr, indx, iA, vA, x, y,
                           ref_y);
}

int ref_make_kronmult_data_f32(int d, int n, int rows, int terms, int mats,
                               int *pntr, int *indx, int *iA, float *vA,
                               float *x, float *y, float *ref_y)
{
  return make_data<float>(d, n, rows, terms, mats, pntr, indx, iA, vA, x, y,
                          ref_y);
}

int ref_make_welem_f64(int d, int n, int terms, int range, int want_ref,
                       int *elem, double *coeff, double *x, double *y,
                       double *ref_y)
{
  return make_welem<double>(d, n, terms, range, want_ref, elem, coeff, x, y, ref_y);
}

int ref_make_welem_f32(int d, int n, int terms, int range, int want_ref,
                       int *elem, float *coeff, float *x, float *y,
                       float *ref_y)
{
  return make_welem<float>(d, n, terms, range, want_ref, elem, coeff, x, y, ref_y);
}

int ref_dense_apply_f64(int d, int n, int rows, int cols, int terms,
                        double const *coeff, int const *elem, int elem_len,
                        int row_offset, int col_offset, int nb, double alpha,
                        double const *x, double beta, double *y)
{
  return dense_apply<double>(d, n, rows, cols, terms, coeff, elem, elem_len,
                             row_offset, col_offset, nb, alpha, x, beta, y);
}

int ref_dense_apply_f32(int d, int n, int rows, int cols, int terms,
                        float const *coeff, int const *elem, int elem_len,
                        int row_offset, int col_offset, int nb, float alpha,
                        float const *x, float beta, float *y)
{
  return dense_apply<float>(d, n, rows, cols, terms, coeff, elem, elem_len,
                            row_offset, col_offset, nb, alpha, x, beta, y);
}

} // extern "C"
