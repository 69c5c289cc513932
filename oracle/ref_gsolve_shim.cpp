// Test infrastructure and the bench's reference arm (never linked by the
// product): the reference's own global-Kronecker implicit solve, end to end,
// compiled from the reference's sources in KRON_MODE_GLOBAL by
// `make -C oracle ref_gsolve` into oracle/_ref/libasgard_ref_gsolve.so.
//
// Everything numerical below is the reference's code, unchanged:
//   * sparse-grid element table      adapt::distributed_grid (src/adapt.cpp,
//                                    src/elements.cpp:248-351)
//   * global patterns, permutations  make_global_kron_matrix
//                                    (src/asgard_kronmult_matrix.cpp:1196-1313)
//   * values + diagonal precond.     set_specific_mode / build_preconditioner
//                                    (src/asgard_kronmult_matrix.cpp:1015-1067,
//                                    1315-1395)
//   * the operator                   global_kron_matrix<P>::apply, CPU branch
//                                    (src/asgard_kronmult_matrix.cpp:1526-1588,
//                                    kronmult::global_cpu)
//   * the solve                      solver::simple_gmres_euler for
//                                    global_kron_matrix (src/solver.cpp:93-117,
//                                    left diagonal preconditioner, CGS GMRES
//                                    :157-298)
//   * workspaces                     matrix_list<P>::make (.hpp:1098-1117)
//
// Two kinds of operator:
//   * ref_gsolve_create_synthetic -- the benchmark's synthetic operator: a
//     PDE<double> of d dimensions and T terms declared through the
//     reference's PDE API (term t acts in dimension t % d with a `div`
//     partial term; every other dimension of a term is the reference's
//     identity `mass` term, which make_global_kron_matrix skips).  Each active
//     term's 1D operator matrix is set through PDE::set_coefficients
//     (src/pde/pde_base.hpp:772-780) from the level-7 3x3 blocks that the
//     reference generated for continuity_1 (term 0, even t) and diffusion_1
//     (term 0, odd t, scaled by nu); identity dimensions keep the eye()
//     matrices the PDE constructor installs (pde_base.hpp:609-611).
//   * ref_gsolve_create_builtin -- a built-in reference PDE by name
//     (make_PDE + generate_all_coefficients), as the reference's driver sets
//     one up for an implicit global-kron run.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

#include "asgard_kronmult_matrix.hpp"
#include "basis.hpp"
#include "coefficients.hpp"
#include "solver.hpp"

using namespace asgard;

namespace
{
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

fk::vector<double> zero_ic(fk::vector<double> const &x, double const)
{
  return fk::vector<double>(x.size());
}

double unit_dt(dimension<double> const &) { return 1.0; }

// d dimensions on [0, 1], all at `level`, degree n (the reference's
// "degree" is the number of polynomial terms per cell).
std::vector<dimension<double>> make_dims(int d, int level, int n)
{
  std::vector<dimension<double>> dims;
  for (int k = 0; k < d; k++)
    dims.emplace_back(0.0, 1.0, level, n, zero_ic, nullptr,
                      "x" + std::to_string(k));
  return dims;
}

term_set<double> make_terms(int d, int T)
{
  term_set<double> terms;
  for (int t = 0; t < T; t++)
  {
    std::vector<term<double>> row;
    for (int k = 0; k < d; k++)
    {
      if (k == t % d)
        row.push_back(term<double>(
            false, "A" + std::to_string(t),
            {partial_term<double>(coefficient_type::div, nullptr, nullptr,
                                  flux_type::upwind,
                                  boundary_condition::periodic,
                                  boundary_condition::periodic)}));
      else
        row.push_back(term<double>(false, "I",
                                   {partial_term<double>(coefficient_type::mass)}));
    }
    terms.push_back(std::move(row));
  }
  return terms;
}

class synthetic_pde : public PDE<double>
{
public:
  synthetic_pde(parser const &cli, int d, int T, int level, int n)
      : PDE<double>(cli, d, 0, T, make_dims(d, level, n), make_terms(d, T),
                    std::vector<source<double>>{},
                    std::vector<md_func_type<double>>{}, nullptr, unit_dt,
                    false, false, std::vector<moment<double>>{}, false)
  {}
};

parser make_cli(std::string const &pde_name, int d, int level, int n)
{
  std::string levels;
  for (int k = 0; k < d; k++)
    levels += (k ? " " : "") + std::to_string(level);
  std::vector<std::string> args = {"-p", pde_name, "-l", levels,
                                   "-d", std::to_string(n), "--kron-mode",
                                   "sparse", "-i", "-s", "gmres"};
  std::vector<char const *> cargs = {"asgard"};
  for (auto &a : args)
    cargs.push_back(a.c_str());
  return parser(static_cast<int>(cargs.size()), cargs.data());
}

struct ref_gsolve
{
  std::unique_ptr<PDE<double>> pde;
  std::unique_ptr<options> opts;
  std::unique_ptr<adapt::distributed_grid<double>> grid;
  matrix_list<double> mats;
  int64_t N = 0;
  int d = 0, n = 0;
};

void finish(ref_gsolve &h)
{
  h.grid = std::make_unique<adapt::distributed_grid<double>>(*h.pde, *h.opts);
  h.mats.make(matrix_entry::regular, *h.pde, *h.grid, *h.opts);
  h.d = h.pde->num_dims;
  h.n = h.pde->get_dimensions()[0].get_degree();
  int64_t ts = 1;
  for (int k = 0; k < h.d; k++)
    ts *= h.n;
  h.N = int64_t(h.grid->get_table().size()) * ts;
}
} // namespace

extern "C"
{
int ref_gsolve_num_threads() { return omp_get_max_threads(); }

// The benchmark operator (see the file header).  pntr7/indx7: the level-7 1D
// connectivity the blocks are stored by (CSR over 1D cells, 2^7 rows);
// adv/dif: one column-major n x n block per level-7 connection.  Returns
// nullptr on bad input.
void *ref_gsolve_create_synthetic(int d, int level, int T, int n, double nu,
                                  int const *pntr7, int const *indx7,
                                  double const *adv, double const *dif)
{
  try
  {
    if (d < 1 || d > 6 || level < 1 || level > 7 || T < 1 || n < 1)
      return nullptr;
    quiet_cout q(true);
    parser const cli = make_cli("continuity_6", d, level, n);
    auto h   = std::make_unique<ref_gsolve>();
    h->pde   = std::make_unique<synthetic_pde>(cli, d, T, level, n);
    h->opts  = std::make_unique<options>(cli);
    int const R  = 1 << level;
    int const nr = n * R;
    for (int t = 0; t < T; t++)
    {
      fk::matrix<double> M(nr, nr); // zero outside connected cells
      connect_1d const cells(level);
      for (int r = 0; r < R; r++)
        for (int j = cells.row_begin(r); j < cells.row_end(r); j++)
        {
          int const c = cells[j];
          // the same connection's block in the level-7 storage
          int pos = -1;
          for (int q7 = pntr7[r]; q7 < pntr7[r + 1]; q7++)
            if (indx7[q7] == c)
              pos = q7;
          if (pos < 0)
            return nullptr;
          double const *b = ((t % 2) == 0 ? adv : dif) + int64_t(pos) * n * n;
          for (int jj = 0; jj < n; jj++)
            for (int i = 0; i < n; i++)
              M(r * n + i, c * n + jj) =
                  (t % 2 == 0) ? b[i + jj * n] : b[i + jj * n] * nu;
        }
      h->pde->set_coefficients(M, t, t % d);
    }
    finish(*h);
    return h.release();
  }
  catch (std::exception const &e)
  {
    std::cerr << "ref_gsolve_create_synthetic: " << e.what() << "\n";
    return nullptr;
  }
}

// A built-in reference PDE (e.g. "continuity_2") at uniform `level`.
void *ref_gsolve_create_builtin(char const *name, int d, int level, int n)
{
  try
  {
    quiet_cout q(true);
    parser const cli = make_cli(name, d, level, n);
    auto h   = std::make_unique<ref_gsolve>();
    h->pde   = make_PDE<double>(cli);
    h->opts  = std::make_unique<options>(cli);
    basis::wavelet_transform<double, resource::host> const transformer(
        *h->opts, *h->pde);
    generate_all_coefficients(*h->pde, transformer);
    finish(*h);
    return h.release();
  }
  catch (std::exception const &e)
  {
    std::cerr << "ref_gsolve_create_builtin: " << e.what() << "\n";
    return nullptr;
  }
}

void ref_gsolve_destroy(void *h) { delete static_cast<ref_gsolve *>(h); }

// d, n, cells, unknowns
int ref_gsolve_info(void *hv, int *d, int *n, int *cells, int64_t *N)
{
  auto *h = static_cast<ref_gsolve *>(hv);
  *d      = h->d;
  *n      = h->n;
  *cells  = h->grid->get_table().size();
  *N      = h->N;
  return 0;
}

// Element table (2*d ints per cell: levels then positions), as the
// reference's grid holds it.
int ref_gsolve_table(void *hv, int *table)
{
  auto *h       = static_cast<ref_gsolve *>(hv);
  auto const &t = h->grid->get_table().get_active_table();
  std::copy_n(t.data(), t.size(), table);
  return 0;
}

// The reference's diagonal preconditioner values pc (z_i = v_i/(1-dt pc_i)).
int ref_gsolve_precond(void *hv, double *pc)
{
  auto *h        = static_cast<ref_gsolve *>(hv);
  auto const &p  = h->mats.kglobal.get_diagonal_preconditioner<resource::host>();
  if (static_cast<int64_t>(p.size()) != h->N)
    return 2;
  std::copy(p.begin(), p.end(), pc);
  return 0;
}

// y = beta*y + alpha*K*x through global_kron_matrix::apply (host).
int ref_gsolve_apply(void *hv, double alpha, double const *x, double beta,
                     double *y, double *seconds)
{
  auto *h = static_cast<ref_gsolve *>(hv);
  try
  {
    auto const t0 = std::chrono::steady_clock::now();
    h->mats.kglobal.apply<resource::host>(matrix_entry::regular, alpha, x,
                                          beta, y);
    if (seconds)
      *seconds = std::chrono::duration<double>(
                     std::chrono::steady_clock::now() - t0)
                     .count();
  }
  catch (std::exception const &)
  {
    return 1;
  }
  return 0;
}

// solver::simple_gmres_euler(dt, matrix_entry::regular, kglobal, x, b,
// restart, max_iter, tol) on host vectors; x is the initial guess and the
// result.  *seconds: wall time of the solver call alone.
int ref_gsolve_gmres_euler(void *hv, double dt, double *x, double const *b,
                           int restart, int max_iter, double tol, int quiet,
                           double *err, int *iters, double *seconds)
{
  auto *h = static_cast<ref_gsolve *>(hv);
  try
  {
    int64_t const N = h->N;
    fk::vector<double> fx(std::vector<double>(x, x + N));
    fk::vector<double> fb(std::vector<double>(b, b + N));
    quiet_cout q(quiet != 0);
    auto const t0 = std::chrono::steady_clock::now();
    auto info = solver::simple_gmres_euler<double, resource::host>(
        dt, matrix_entry::regular, h->mats.kglobal, fx, fb, restart, max_iter,
        tol);
    if (seconds)
      *seconds = std::chrono::duration<double>(
                     std::chrono::steady_clock::now() - t0)
                     .count();
    std::copy_n(fx.data(), N, x);
    *err   = info.error;
    *iters = info.iterations;
  }
  catch (std::exception const &e)
  {
    std::cerr << "ref_gsolve_gmres_euler: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
} // extern "C"
