// C++ mirror of the reference's kronmult_matrix<P> and simple_gmres_euler
// (src/asgard_kronmult_matrix.hpp:111-682, src/solver.hpp:17-41) over the C
// ABI of asgard_b200.h.  Header-only; link libasgard_b200.so.
//
// Differences from the reference types: vectors are std::vector (host) or raw
// device pointers instead of fk::vector.  P = double and P = float are
// provided, as the reference instantiates them (ASGARD_ENABLE_DOUBLE /
// ASGARD_ENABLE_FLOAT, src/asgard_kronmult_matrix.cpp:1620-1640); a float
// matrix keeps its factors as given (the plan also holds them widened to
// FP64), applies device vectors in FP32 and host vectors through the FP64
// host path.  Errors raise the
// reference's exception types: std::runtime_error, and std::invalid_argument
// for a restart larger than the system (src/solver.cpp:175-181).
#pragma once

#include "asgard_b200.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace asgard_b200
{
enum class resource
{
  host,
  device
};

//! gmres_info<P> of src/pde/pde_base.hpp:93-97
template<typename P>
struct gmres_info
{
  P error;
  int iterations;
};

inline void check(int status, char const *what)
{
  if (status != ASGK_OK)
    throw std::runtime_error(std::string(what) + ": " + asgk_status_string(status));
}

namespace detail
{
//! factors and vectors handed to the C ABI, which takes FP64 host arrays
template<typename P>
std::vector<double> widen(std::vector<P> const &v)
{
  return std::vector<double>(v.begin(), v.end());
}
inline std::vector<double> const &widen(std::vector<double> const &v) { return v; }
} // namespace detail

template<typename P>
class kronmult_matrix
{
  static_assert(std::is_same_v<P, double> || std::is_same_v<P, float>,
                "kronmult_matrix<P>: P is double or float");

public:
  kronmult_matrix() = default;

  //! Sparse CPU form (src/asgard_kronmult_matrix.hpp:284-297, one chunk):
  //! CSR over output cells, per-pair factor offsets iA into vA.
  kronmult_matrix(int num_dimensions, int kron_size, int num_rows,
                  int num_cols, int num_terms, std::vector<int> const &pntr,
                  std::vector<int> const &indx, std::vector<int> const &iA,
                  std::vector<P> const &vA)
      : d_(num_dimensions), n_(kron_size), rows_(num_rows), cols_(num_cols),
        terms_(num_terms)
  {
    if (pntr.size() != size_t(num_rows) + 1)
      throw std::runtime_error("kronmult_matrix: pntr must have num_rows + 1 entries");
    std::vector<int64_t> rp(pntr.begin(), pntr.end());
    auto const &wv = detail::widen(vA);
    check(asgk_plan_create(&plan_, d_, n_, rows_, cols_, terms_, rp.data(),
                           indx.data(), iA.data(), wv.data(),
                           int64_t(wv.size())),
          "kronmult_matrix");
  }

  //! Multi-call CPU form (src/asgard_kronmult_matrix.hpp:284-297, 580-627):
  //! consecutive blocks of output rows, chunk i a CSR over its own rows
  //! (list_pntr[i] has rows_i + 1 entries, sum rows_i = num_rows) with its
  //! iA.  The reference applies the chunks one call each (the split bounds
  //! its 32-bit offsets); here they form one plan, the same operator.
  kronmult_matrix(int num_dimensions, int kron_size, int num_rows,
                  int num_cols, int num_terms,
                  std::vector<std::vector<int>> const &list_pntr,
                  std::vector<std::vector<int>> const &list_indx,
                  std::vector<std::vector<int>> const &list_iA,
                  std::vector<P> const &vA)
      : d_(num_dimensions), n_(kron_size), rows_(num_rows), cols_(num_cols),
        terms_(num_terms)
  {
    if (list_pntr.size() != list_indx.size() || list_pntr.size() != list_iA.size())
      throw std::runtime_error("kronmult_matrix: chunk lists differ in length");
    std::vector<int64_t> rp(1, 0);
    std::vector<int> indx, iA;
    for (size_t c = 0; c < list_pntr.size(); c++)
    {
      auto const &p = list_pntr[c];
      if (p.empty() || p.front() != 0 || size_t(p.back()) != list_indx[c].size())
        throw std::runtime_error("kronmult_matrix: bad chunk row pointers");
      int64_t const base = rp.back();
      for (size_t r = 1; r < p.size(); r++)
        rp.push_back(base + p[r]);
      indx.insert(indx.end(), list_indx[c].begin(), list_indx[c].end());
      iA.insert(iA.end(), list_iA[c].begin(), list_iA[c].end());
    }
    if (rp.size() != size_t(num_rows) + 1)
      throw std::runtime_error("kronmult_matrix: chunks must cover num_rows rows");
    auto const &wv = detail::widen(vA);
    check(asgk_plan_create(&plan_, d_, n_, rows_, cols_, terms_, rp.data(),
                           indx.data(), iA.data(), wv.data(),
                           int64_t(wv.size())),
          "kronmult_matrix");
  }

  //! Multi-call GPU form (src/asgard_kronmult_matrix.hpp:284-297, 372-449):
  //! chunks of pairs in the GPU format, all acting on the whole of y (beta
  //! once, as the reference passes it to the first chunk only).
  static kronmult_matrix from_pair_lists(int num_dimensions, int kron_size,
                                         int num_rows, int num_cols, int num_terms,
                                         std::vector<std::vector<int>> const &list_row_indx,
                                         std::vector<std::vector<int>> const &list_col_indx,
                                         std::vector<std::vector<int>> const &list_iA,
                                         std::vector<P> const &vA)
  {
    if (list_row_indx.size() != list_col_indx.size() ||
        list_row_indx.size() != list_iA.size())
      throw std::runtime_error("kronmult_matrix: chunk lists differ in length");
    std::vector<int> ri, ci, ia;
    for (size_t c = 0; c < list_row_indx.size(); c++)
    {
      ri.insert(ri.end(), list_row_indx[c].begin(), list_row_indx[c].end());
      ci.insert(ci.end(), list_col_indx[c].begin(), list_col_indx[c].end());
      ia.insert(ia.end(), list_iA[c].begin(), list_iA[c].end());
    }
    return from_pairs(num_dimensions, kron_size, num_rows, num_cols, num_terms,
                      ri, ci, ia, vA);
  }

  //! Sparse GPU form (src/asgard_kronmult_matrix.hpp:235-272): per pair the
  //! tensor offsets into y (row_indx) and x (col_indx).
  static kronmult_matrix from_pairs(int num_dimensions, int kron_size,
                                    int num_rows, int num_cols, int num_terms,
                                    std::vector<int> const &row_indx,
                                    std::vector<int> const &col_indx,
                                    std::vector<int> const &iA,
                                    std::vector<P> const &vA)
  {
    kronmult_matrix m;
    m.d_     = num_dimensions;
    m.n_     = kron_size;
    m.rows_  = num_rows;
    m.cols_  = num_cols;
    m.terms_ = num_terms;
    if (row_indx.size() != col_indx.size())
      throw std::runtime_error("kronmult_matrix: row/col index sizes differ");
    check(asgk_plan_create_pairs(&m.plan_, m.d_, m.n_, m.rows_, m.cols_,
                                 m.terms_, int64_t(row_indx.size()),
                                 row_indx.data(), col_indx.data(), iA.data(),
                                 detail::widen(vA).data(), int64_t(vA.size())),
          "kronmult_matrix");
    return m;
  }

  //! Dense form (src/asgard_kronmult_matrix.hpp:132-176): every output cell
  //! with every input cell; terms[t] holds d * num_1d_blocks^2 column-major
  //! n x n blocks (per dimension ordered by column cell, then row cell, as
  //! make_kronmult_dense writes them), elem the d 1D cell indices of every
  //! cell; rows start at elem entry row_offset, columns at col_offset.
  kronmult_matrix(int num_dimensions, int kron_size, int num_rows,
                  int num_cols, int num_terms,
                  std::vector<std::vector<P>> const &terms,
                  std::vector<int> const &elem, int row_offset, int col_offset,
                  int num_1d_blocks)
      : d_(num_dimensions), n_(kron_size), rows_(num_rows), cols_(num_cols),
        terms_(num_terms)
  {
    if (terms.size() != size_t(num_terms))
      throw std::runtime_error("kronmult_matrix: terms must hold num_terms arrays");
    std::vector<std::vector<double>> wide;
    std::vector<double const *> tp;
    for (auto const &t : terms)
    {
      wide.push_back(detail::widen(t));
      tp.push_back(wide.back().data());
    }
    check(asgk_plan_create_dense(&plan_, d_, n_, rows_, cols_, terms_,
                                 tp.data(), elem.data(), int64_t(elem.size()),
                                 row_offset, col_offset, num_1d_blocks),
          "kronmult_matrix");
  }

  //! Global Kronecker form of a sparse-grid operator (the reference's
  //! global_kron_matrix, src/asgard_kronmult_matrix.cpp:1196-1334): the
  //! element table (num_cells x 2d levels then positions, asgk_sparse_grid's
  //! layout) and the factors per 1D connection (asgk_plan_create_conn's
  //! layout).  Terms acting in one dimension are applied in one pass, terms
  //! acting in several by the reference's upper/lower permutations.
  static kronmult_matrix global_form(int num_dimensions, int kron_size,
                                     int level, std::vector<int> const &table,
                                     int num_terms,
                                     std::vector<P> const &vA)
  {
    kronmult_matrix m;
    int const cells = int(table.size() / (2 * size_t(num_dimensions)));
    m.d_     = num_dimensions;
    m.n_     = kron_size;
    m.rows_  = cells;
    m.cols_  = cells;
    m.terms_ = num_terms;
    check(asgk_plan_create_global(&m.plan_, num_dimensions, kron_size, level,
                                  cells, table.data(), num_terms,
                                  detail::widen(vA).data(), int64_t(vA.size())),
          "kronmult_matrix");
    return m;
  }

  kronmult_matrix(kronmult_matrix const &) = delete;
  kronmult_matrix &operator=(kronmult_matrix const &) = delete;
  kronmult_matrix(kronmult_matrix &&o) noexcept { swap(o); }
  kronmult_matrix &operator=(kronmult_matrix &&o) noexcept
  {
    swap(o);
    return *this;
  }
  ~kronmult_matrix() { asgk_plan_destroy(plan_); }

  //! y = beta*y + alpha*K*x; rec says where x and y live
  //! (src/asgard_kronmult_matrix.hpp:340-478).  Not thread-safe, as there.
  template<resource rec = resource::host>
  void apply(P alpha, P const x[], P beta, P y[]) const
  {
    if constexpr (std::is_same_v<P, double>)
    {
      if constexpr (rec == resource::host)
        check(asgk_apply_host(plan_, alpha, x, beta, y, nullptr), "apply");
      else
        check(asgk_apply(plan_, ASGK_FP64, alpha, x, beta, y, nullptr), "apply");
    }
    else if constexpr (rec == resource::device)
      check(asgk_apply_f32(plan_, alpha, x, beta, y, nullptr), "apply");
    else
    {
      std::vector<double> xd(x, x + input_size()), yd(y, y + output_size());
      check(asgk_apply_host(plan_, alpha, xd.data(), beta, yd.data(), nullptr),
            "apply");
      for (size_t i = 0; i < yd.size(); i++)
        y[i] = P(yd[i]);
    }
  }

  //! num_rows * num_cols, as the reference returns for every matrix
  //! (src/asgard_kronmult_matrix.hpp:481)
  int64_t num_batch() const { return int64_t(rows_) * int64_t(cols_); }
  //! the (row, col) products one apply computes (stored pairs)
  int64_t num_pairs() const { return info(0); }
  int tensor_size() const { return compute_tensor_size(d_, n_); }
  int input_size() const { return int(info(1)); }
  int output_size() const { return int(info(2)); }
  //! as the reference's flops(): n^d * n * |iA| (multiply-add counted once)
  int64_t flops() const { return info(3) / 2; }
  explicit operator bool() const { return d_ > 0; }
  bool is_dense() const { return plan_ != nullptr && asgk_plan_kind(plan_) == 1; }
  bool is_onecall() const { return true; }
  //! device buffers for apply<resource::host> (src/asgard_kronmult_matrix.hpp:301-307)
  void set_workspace(double *xdev, double *ydev)
  {
    check(asgk_plan_set_workspace(plan_, xdev, input_size(), ydev, output_size()),
          "set_workspace");
  }

  static int compute_tensor_size(int num_dimensions, int kron_size)
  {
    int t = kron_size;
    for (int i = 1; i < num_dimensions; i++)
      t *= kron_size;
    return t;
  }
  static int64_t compute_flops(int num_dimensions, int kron_size,
                               int num_terms, int64_t num_batch)
  {
    return int64_t(compute_tensor_size(num_dimensions, kron_size)) *
           kron_size * num_dimensions * num_terms * num_batch * 2;
  }

  void update_stored_coefficients(std::vector<P> const &vA)
  {
    check(asgk_plan_update_values(plan_, detail::widen(vA).data(), int64_t(vA.size())),
          "update_stored_coefficients");
  }
  //! dense matrices: new per-term arrays (src/asgard_kronmult_matrix.hpp:538-561)
  void update_stored_coefficients(std::vector<std::vector<P>> const &terms)
  {
    std::vector<std::vector<double>> wide;
    std::vector<double const *> tp;
    for (auto const &t : terms)
    {
      wide.push_back(detail::widen(t));
      tp.push_back(wide.back().data());
    }
    check(asgk_plan_update_terms(plan_, tp.data(), int(terms.size())),
          "update_stored_coefficients");
  }

  asgk_plan *plan() const { return plan_; }

private:
  int64_t info(int which) const
  {
    int64_t v[5] = {0, 0, 0, 0, 0};
    check(asgk_plan_info(plan_, &v[0], &v[1], &v[2], &v[3], &v[4]), "info");
    return v[which];
  }
  void swap(kronmult_matrix &o) noexcept
  {
    std::swap(plan_, o.plan_);
    std::swap(d_, o.d_);
    std::swap(n_, o.n_);
    std::swap(rows_, o.rows_);
    std::swap(cols_, o.cols_);
    std::swap(terms_, o.terms_);
  }

  asgk_plan *plan_ = nullptr;
  int d_ = 0, n_ = 0, rows_ = 0, cols_ = 0, terms_ = 0;
};

namespace solver
{
//! Solves (I - dt*K) x = b on device vectors (x holds the initial guess),
//! the reference's criterion (absolute tolerance on the estimated residual)
//! -- src/solver.cpp:119-135.
inline gmres_info<double>
simple_gmres_euler(double dt, kronmult_matrix<double> const &mat, double *x,
                   double const *b, int restart, int max_iter, double tol)
{
  int64_t const n = mat.output_size();
  if (restart > n)
    throw std::invalid_argument("Number of inner iterations " +
                                std::to_string(restart) + " must be less than " +
                                std::to_string(n) + "!");
  asgk_gmres_info info{};
  check(asgk_gmres_euler(mat.plan(), dt, x, b, restart, max_iter, tol,
                         ASGK_TOL_ABS, ASGK_FP64, nullptr, &info, nullptr),
        "simple_gmres_euler");
  if (info.status == ASGK_ERR_NONFINITE)
    throw std::runtime_error("simple_gmres_euler: non-finite residual");
  return gmres_info<double>{info.error, info.iterations};
}

//! The same for kronmult_matrix<float> on FP32 device vectors (the
//! reference's FP32 instantiation): solved with the FP32 operator inside
//! FP64 iterative refinement on FP64 copies (asgk_gmres_euler_f32), the
//! reference's absolute criterion applied to the FP64 residual.
inline gmres_info<float>
simple_gmres_euler(float dt, kronmult_matrix<float> const &mat, float *x,
                   float const *b, int restart, int max_iter, float tol)
{
  int64_t const n = mat.output_size();
  if (restart > n)
    throw std::invalid_argument("Number of inner iterations " +
                                std::to_string(restart) + " must be less than " +
                                std::to_string(n) + "!");
  asgk_gmres_info info{};
  check(asgk_gmres_euler_f32(mat.plan(), dt, x, b, restart, max_iter, tol, &info,
                             nullptr),
        "simple_gmres_euler");
  if (info.status == ASGK_ERR_NONFINITE)
    throw std::runtime_error("simple_gmres_euler: non-finite residual");
  return gmres_info<float>{float(info.error), info.iterations};
}

//! A Jacobi preconditioner of I - dt*K built on the device and owned here:
//! ASGK_JACOBI_POINT is the reference's diagonal preconditioner
//! (build_preconditioner, src/asgard_kronmult_matrix.cpp:1015-1067);
//! ASGK_JACOBI_BLOCK and ASGK_JACOBI_KRON invert each cell's diagonal block
//! (KRON: global plans whose terms act in one dimension each, any d).
class jacobi_preconditioner
{
public:
  jacobi_preconditioner(kronmult_matrix<double> const &mat, double dt,
                        int kind = ASGK_JACOBI_POINT)
      : dt_(dt)
  {
    check(asgk_jacobi_create(&pc_, mat.plan(), dt, kind), "jacobi_preconditioner");
  }
  ~jacobi_preconditioner()
  {
    if (pc_)
      asgk_jacobi_destroy(pc_);
  }
  jacobi_preconditioner(jacobi_preconditioner const &)            = delete;
  jacobi_preconditioner &operator=(jacobi_preconditioner const &) = delete;
  jacobi_preconditioner(jacobi_preconditioner &&o) noexcept
      : pc_(std::exchange(o.pc_, nullptr)), dt_(o.dt_)
  {}
  jacobi_preconditioner &operator=(jacobi_preconditioner &&o) noexcept
  {
    std::swap(pc_, o.pc_);
    std::swap(dt_, o.dt_);
    return *this;
  }
  asgk_jacobi *handle() const { return pc_; }
  double dt() const { return dt_; }

private:
  asgk_jacobi *pc_ = nullptr;
  double dt_       = 0;
};

//! The counterpart of the reference's global-kron simple_gmres_euler, which
//! preconditions with its diagonal preconditioner (src/solver.cpp:93-117):
//! here the caller's Jacobi preconditioner of (mat, dt) is applied on the
//! right through flexible GMRES, so the solve stops on the estimate of the
//! unpreconditioned residual (absolute tolerance), whereas the reference
//! applies its preconditioner on the left and stops on the preconditioned
//! residual; iteration counts and the returned error therefore differ from
//! the reference's.  A preconditioner built for another step size than dt
//! is refused (std::invalid_argument).
inline gmres_info<double>
simple_gmres_euler(double dt, kronmult_matrix<double> const &mat, double *x,
                   double const *b, int restart, int max_iter, double tol,
                   jacobi_preconditioner const &pc)
{
  if (pc.dt() != dt)
    throw std::invalid_argument("simple_gmres_euler: the preconditioner was built for dt = " +
                                std::to_string(pc.dt()) + ", not " + std::to_string(dt));
  int64_t const n = mat.output_size();
  if (restart > n)
    throw std::invalid_argument("Number of inner iterations " +
                                std::to_string(restart) + " must be less than " +
                                std::to_string(n) + "!");
  asgk_gmres_info info{};
  check(asgk_gmres_euler_jacobi(mat.plan(), dt, x, b, restart, max_iter, tol,
                                ASGK_TOL_ABS, ASGK_FP64, pc.handle(), &info,
                                nullptr),
        "simple_gmres_euler");
  if (info.status == ASGK_ERR_NONFINITE)
    throw std::runtime_error("simple_gmres_euler: non-finite residual");
  return gmres_info<double>{info.error, info.iterations};
}

//! solver::simple_gmres on a dense column-major host matrix with the
//! reference's dense preconditioner M (src/solver.cpp:11-38, 55-74): M
//! (column-major n x n) is LU-factored and applied on the left; an empty M
//! means none, as an empty fk::matrix does there.
inline gmres_info<double> simple_gmres(std::vector<double> const &A,
                                       std::vector<double> &x,
                                       std::vector<double> const &b,
                                       std::vector<double> const &M,
                                       int restart, int max_iter, double tol)
{
  int const n = int(b.size());
  if (restart > n)
    throw std::invalid_argument("Number of inner iterations " +
                                std::to_string(restart) + " must be less than " +
                                std::to_string(n) + "!");
  if (A.size() != size_t(n) * n || x.size() != size_t(n) ||
      (!M.empty() && M.size() != size_t(n) * n))
    throw std::runtime_error("simple_gmres: A, x, b and M sizes differ");
  asgk_gmres_info info{};
  check(asgk_gmres_dense_precond(n, A.data(), x.data(), b.data(),
                                 M.empty() ? nullptr : M.data(), restart,
                                 max_iter, tol, &info),
        "simple_gmres");
  return gmres_info<double>{info.error, info.iterations};
}

//! The same without a preconditioner.
inline gmres_info<double> simple_gmres(std::vector<double> const &A,
                                       std::vector<double> &x,
                                       std::vector<double> const &b,
                                       int restart, int max_iter, double tol)
{
  return simple_gmres(A, x, b, std::vector<double>(), restart, max_iter, tol);
}
} // namespace solver
} // namespace asgard_b200
