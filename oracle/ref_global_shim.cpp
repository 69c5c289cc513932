// Test infrastructure (CPU baseline and checker only; compiled with
// KRON_MODE_GLOBAL against the reference sources by `make -C oracle
// ref_global`): drives the reference's fast global Kronecker product,
// kronmult::global_cpu (src/device/asgard_glkronmult_cpu.cpp:150-188),
// on a sparse-grid operator given as element table + per-1D-connection
// factor blocks (the layout of asgk_plan_create_conn).
//
// The inputs global_cpu expects are built here the way
// make_global_kron_matrix does (src/asgard_kronmult_matrix.cpp:1196-1290):
// per dimension a sparsity pattern over all degrees of freedom (a dof's
// columns are the dofs that agree with it in every other dimension and whose
// 1D cell is connected to its own; gdiag marks the diagonal entry), the
// values of every term in its active dimensions, and per term the
// permutations over its active (non-identity) dimensions
// (check_identity_term + permutes::remap_directions, :1293-1312).
#include "asgard_kronmult.hpp"

#include <chrono>
#include <unordered_map>
#include <vector>

namespace
{
int index_1d(int level, int pos) { return level == 0 ? 0 : (1 << (level - 1)) + pos; }
} // namespace

struct ref_global
{
  int d = 0;
  int64_t ndof = 0;
  std::vector<asgard::kronmult::permutes> perms;
  std::vector<std::vector<int>> gpntr, gindx, gdiag;
  std::vector<std::vector<double>> gvals;
  std::vector<int> terms;
  std::vector<double> w1, w2;
};

extern "C"
{
// Builds the global form (host, single thread).  vA: [1D connection][term]
// [dimension][n*n] column-major blocks.  Returns nullptr on bad input.
void *ref_global_create(int d, int n, int level, int num_cells,
                        const int *table, int T, const double *vA)
{
  using namespace asgard;
  if (d < 1 || d > 6 || n < 1 || level < 0 || level > 12 || num_cells < 1 ||
      T < 1)
    return nullptr;
  connect_1d const cells(level); // full hierarchy, as the local mode
  int const R = 1 << level;
  int64_t ts = 1;
  for (int k = 0; k < d; k++)
    ts *= n;
  int64_t const ndof = int64_t(num_cells) * ts;
  // 1D cell of every cell in every dimension
  std::vector<int> c1(size_t(num_cells) * d);
  for (int c = 0; c < num_cells; c++)
    for (int k = 0; k < d; k++)
      c1[size_t(c) * d + k] = index_1d(table[int64_t(c) * 2 * d + k],
                                       table[int64_t(c) * 2 * d + d + k]);
  // 1D dof index of every dof in every dimension: cell * n + polynomial
  auto dof1d = [&](int64_t dof, int k) {
    int64_t const c = dof / ts;
    int64_t e       = dof % ts;
    for (int q = d - 1; q > k; q--)
      e /= n;
    return c1[size_t(c) * d + k] * n + int(e % n);
  };
  int bits = 1;
  while ((int64_t(1) << bits) < int64_t(R) * n)
    ++bits;
  if (bits * d > 64)
    return nullptr;
  auto key = [&](int64_t dof, int kk, int repl) {
    uint64_t h = 0;
    for (int k = 0; k < d; k++)
      h = (h << bits) | uint64_t(k == kk ? repl : dof1d(dof, k));
    return h;
  };
  std::unordered_map<uint64_t, int> where;
  where.reserve(size_t(ndof) * 2);
  for (int64_t g = 0; g < ndof; g++)
    where.emplace(key(g, -1, 0), int(g));

  // active dimensions of each term: not the identity (I at self connections,
  // 0 elsewhere)
  int const nconn = cells.num_connections();
  auto blk = [&](int j, int t, int k) {
    return vA + (int64_t(j) * T + t) * d * n * n + int64_t(k) * n * n;
  };
  std::vector<std::vector<int>> active(T);
  for (int t = 0; t < T; t++)
    for (int k = 0; k < d; k++)
    {
      bool ident = true;
      for (int r = 0; r < R && ident; r++)
        for (int j = cells.row_begin(r); j < cells.row_end(r) && ident; j++)
        {
          const double *a = blk(j, t, k);
          for (int e = 0; e < n * n && ident; e++)
            ident = a[e] == ((cells[j] == r && e % (n + 1) == 0) ? 1.0 : 0.0);
        }
      if (!ident)
        active[t].push_back(k);
    }
  (void)nconn;

  std::vector<std::vector<int>> gpntr(d), gindx(d), gdiag(d);
  std::vector<std::vector<double>> gvals(size_t(T) * d);
  for (int k = 0; k < d; k++)
  {
    auto &pntr = gpntr[k];
    auto &indx = gindx[k];
    auto &diag = gdiag[k];
    pntr.assign(ndof + 1, 0);
    diag.assign(ndof, 0);
    std::vector<int> cconn; // cell-level connection of every entry
    for (int64_t g = 0; g < ndof; g++)
    {
      int const rk = dof1d(g, k);
      int const rc = rk / n;
      for (int j = cells.row_begin(rc); j < cells.row_end(rc); j++)
        for (int p = 0; p < n; p++)
        {
          auto it = where.find(key(g, k, cells[j] * n + p));
          if (it == where.end())
            continue;
          if (it->second == g)
            diag[g] = int(indx.size());
          indx.push_back(it->second);
          cconn.push_back(j * n * n + p * n + rk % n); // A(row poly, col poly)
        }
      pntr[g + 1] = int(indx.size());
    }
    for (int t = 0; t < T; t++)
    {
      bool act = false;
      for (int a : active[t])
        act = act || (a == k);
      if (!act)
        continue;
      auto &v = gvals[size_t(t) * d + k];
      v.resize(indx.size());
      for (size_t e = 0; e < indx.size(); e++)
      {
        int const j  = cconn[e] / (n * n);
        int const pc = (cconn[e] / n) % n, pr = cconn[e] % n;
        v[e]         = blk(j, t, k)[pr + pc * n];
      }
    }
  }
  auto *g = new ref_global();
  g->d    = d;
  g->ndof = ndof;
  for (int t = 0; t < T; t++)
  {
    g->perms.emplace_back(int(active[t].size()));
    g->perms.back().remap_directions(active[t]);
    g->terms.push_back(t);
  }
  g->gpntr = std::move(gpntr);
  g->gindx = std::move(gindx);
  g->gdiag = std::move(gdiag);
  g->gvals = std::move(gvals);
  g->w1.assign(ndof, 0.0);
  g->w2.assign(ndof, 0.0);
  return g;
}

// y = K x (y overwritten) `reps` times; *seconds = the best time of one
// product (global_cpu, OpenMP on all threads).
int ref_global_run(void *handle, int reps, const double *x, double *y,
                   double *seconds)
{
  auto *g = static_cast<ref_global *>(handle);
  if (!g || reps < 1)
    return -1;
  double best = 1e300;
  for (int rep = 0; rep < reps; rep++)
  {
    std::fill(y, y + g->ndof, 0.0);
    auto const t0 = std::chrono::steady_clock::now();
    asgard::kronmult::global_cpu(g->d, g->perms, g->gpntr, g->gindx, g->gdiag,
                                 g->gvals, g->terms, x, y, g->w1.data(),
                                 g->w2.data());
    double const s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    best = std::min(best, s);
  }
  if (seconds)
    *seconds = best;
  return 0;
}

void ref_global_destroy(void *handle) { delete static_cast<ref_global *>(handle); }
} // extern "C"
