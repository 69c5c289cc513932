// Drives the C++ drop-in header (include/asgard_b200/kronmult_matrix.hpp) the
// way reference code would: builds a sparse-grid operator (d = 3, level 4,
// 2 terms, seeded random factors) in the reference's CPU CSR format, its
// multi-call chunk forms and its dense form, applies it on host and device
// vectors, solves one backward-Euler step with simple_gmres_euler, repeats
// apply and solve through kronmult_matrix<float>, solves one dense system
// with simple_gmres (with and without the dense preconditioner), and writes
// inputs and results to a binary file for tests/test_cpp_dropin_gpu.py.
#include "asgard_b200/kronmult_matrix.hpp"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <fstream>
#include <random>
#include <vector>

using namespace asgard_b200;

template<typename T>
void put(std::ofstream &o, std::vector<T> const &v)
{
  int64_t const n = int64_t(v.size());
  o.write(reinterpret_cast<char const *>(&n), sizeof(n));
  o.write(reinterpret_cast<char const *>(v.data()), sizeof(T) * v.size());
}

int main(int argc, char **argv)
{
  if (argc < 2)
    return 2;
  int const d = 3, L = 4, n = 3, T = 2;
  int64_t const cells = asgk_sparse_grid(d, L, nullptr);
  std::vector<int> table(cells * 2 * d);
  asgk_sparse_grid(d, L, table.data());
  int64_t nnz = 0;
  check(asgk_build_pairs(d, L, int(cells), table.data(), &nnz, nullptr,
                         nullptr, nullptr),
        "build_pairs");
  std::vector<int64_t> rp(cells + 1);
  std::vector<int> col(nnz), conn(nnz * d);
  check(asgk_build_pairs(d, L, int(cells), table.data(), &nnz, rp.data(),
                         col.data(), conn.data()),
        "build_pairs");
  int nrows1d = 0, nconn = 0;
  asgk_connect_1d(L, &nrows1d, &nconn, nullptr, nullptr);
  // reference layout: iA = conn*(d*T*n*n) + (t*d + k)*n*n
  std::vector<int> iA(nnz * T * d);
  for (int64_t p = 0; p < nnz; p++)
    for (int t = 0; t < T; t++)
      for (int k = 0; k < d; k++)
        iA[(p * T + t) * d + k] = conn[p * d + k] * d * T * n * n + (t * d + k) * n * n;
  std::mt19937_64 rng(17);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  std::vector<double> vA(int64_t(nconn) * d * T * n * n);
  for (auto &v : vA)
    v = 0.2 * U(rng);
  std::vector<int> pntr(rp.begin(), rp.end());
  kronmult_matrix<double> mat(d, n, int(cells), int(cells), T, pntr, col, iA, vA);
  int const N = mat.output_size();

  std::vector<double> x(N), y_host(N), b(N);
  for (auto &v : x)
    v = U(rng);
  for (auto &v : b)
    v = U(rng);
  for (auto &v : y_host)
    v = U(rng);
  std::vector<double> y0 = y_host;
  mat.apply<resource::host>(0.5, x.data(), -2.0, y_host.data());

  double *dx = nullptr, *dy = nullptr, *db = nullptr;
  cudaMalloc(&dx, sizeof(double) * N);
  cudaMalloc(&dy, sizeof(double) * N);
  cudaMalloc(&db, sizeof(double) * N);
  cudaMemcpy(dx, x.data(), sizeof(double) * N, cudaMemcpyHostToDevice);
  cudaMemcpy(dy, y0.data(), sizeof(double) * N, cudaMemcpyHostToDevice);
  mat.apply<resource::device>(0.5, dx, -2.0, dy);
  std::vector<double> y_dev(N);
  cudaMemcpy(y_dev.data(), dy, sizeof(double) * N, cudaMemcpyDeviceToHost);

  // one implicit step: (I - dt K) sol = b
  cudaMemcpy(db, b.data(), sizeof(double) * N, cudaMemcpyHostToDevice);
  cudaMemset(dx, 0, sizeof(double) * N);
  auto info = solver::simple_gmres_euler(1e-2, mat, dx, db, 20, 50, 1e-12);
  std::vector<double> sol(N);
  cudaMemcpy(sol.data(), dx, sizeof(double) * N, cudaMemcpyDeviceToHost);

  // the same step through the overload of the reference's global-kron
  // simple_gmres_euler, with a diagonal (point Jacobi) preconditioner
  double pc_rel = 1.0, pc_its = 0.0, pc_err = 1.0;
  {
    solver::jacobi_preconditioner pc(mat, 1e-2, ASGK_JACOBI_POINT);
    cudaMemset(dx, 0, sizeof(double) * N);
    auto ip = solver::simple_gmres_euler(1e-2, mat, dx, db, 20, 50, 1e-12, pc);
    std::vector<double> sp(N);
    cudaMemcpy(sp.data(), dx, sizeof(double) * N, cudaMemcpyDeviceToHost);
    double nu = 0, de = 0;
    for (int64_t i = 0; i < N; i++)
    {
      nu += (sp[i] - sol[i]) * (sp[i] - sol[i]);
      de += sol[i] * sol[i];
    }
    pc_rel = std::sqrt(nu / de);
    pc_its = ip.iterations;
    pc_err = ip.error;
  }

  // the same operator in the global Kronecker form (every term here acts in
  // all dimensions: chains of masked 1D passes), then a single-direction
  // operator
  double global_multi_rel = 1.0;
  {
    std::vector<int> tb(table.begin(), table.end());
    auto g = kronmult_matrix<double>::global_form(d, n, L, tb, T, vA);
    std::vector<double> ym(N, 0.0), yq(N, 0.0);
    g.apply<resource::host>(1.0, x.data(), 0.0, ym.data());
    mat.apply<resource::host>(1.0, x.data(), 0.0, yq.data());
    double nu = 0, de = 0;
    for (int i = 0; i < N; i++)
    {
      nu += (ym[i] - yq[i]) * (ym[i] - yq[i]);
      de += yq[i] * yq[i];
    }
    global_multi_rel = std::sqrt(nu / de);
  }
  // advection-like factors in dimension t only (identity elsewhere)
  std::vector<double> vS(vA.size(), 0.0);
  std::vector<int> c1p(nrows1d + 1), c1i(nconn);
  asgk_connect_1d(L, &nrows1d, &nconn, c1p.data(), c1i.data());
  for (int r = 0; r < nrows1d; r++)
    for (int j = c1p[r]; j < c1p[r + 1]; j++)
      for (int t = 0; t < T; t++)
        for (int k = 0; k < d; k++)
          for (int e = 0; e < 9; e++)
          {
            double &v = vS[((int64_t(j) * T + t) * d + k) * 9 + e];
            if (k == t % d)
              v = 0.2 * U(rng);
            else
              v = (c1i[j] == r && e % 4 == 0) ? 1.0 : 0.0;
          }
  std::vector<int> tb(table.begin(), table.end());
  auto gS = kronmult_matrix<double>::global_form(d, n, L, tb, T, vS);
  kronmult_matrix<double> pS(d, n, int(cells), int(cells), T, pntr, col, iA, vS);
  std::vector<double> yg(N), yp(N);
  gS.apply<resource::host>(1.0, x.data(), 0.0, yg.data());
  pS.apply<resource::host>(1.0, x.data(), 0.0, yp.data());
  double num = 0, den = 0;
  for (int i = 0; i < N; i++)
  {
    num += (yg[i] - yp[i]) * (yg[i] - yp[i]);
    den += yp[i] * yp[i];
  }
  double const global_rel = std::sqrt(num / den);

  // the same operator in the reference's dense form (make_kronmult_dense's
  // layout): full 1D operators with the connection blocks, zero elsewhere,
  // and the cells' 1D indices; every (row, col) pair is then computed
  int const nb = nrows1d;
  std::vector<std::vector<double>> dterms(T, std::vector<double>(size_t(d) * nb * nb * 9, 0.0));
  for (int r = 0; r < nrows1d; r++)
    for (int j = c1p[r]; j < c1p[r + 1]; j++)
      for (int t = 0; t < T; t++)
        for (int k = 0; k < d; k++)
          for (int e = 0; e < 9; e++)
            dterms[t][((size_t(k) * nb + c1i[j]) * nb + r) * 9 + e] =
                vA[((int64_t(j) * T + t) * d + k) * 9 + e];
  std::vector<int> elem(size_t(cells) * d);
  for (int64_t c = 0; c < cells; c++)
    for (int k = 0; k < d; k++)
    {
      int const lev = table[c * 2 * d + k], pos = table[c * 2 * d + d + k];
      elem[c * d + k] = (lev == 0) ? 0 : (1 << (lev - 1)) + pos;
    }
  kronmult_matrix<double> dmat(d, n, int(cells), int(cells), T, dterms, elem, 0, 0, nb);
  std::vector<double> y_dense = y0;
  dmat.apply<resource::host>(0.5, x.data(), -2.0, y_dense.data());
  auto rel = [&](std::vector<double> const &a, std::vector<double> const &ref) {
    double nu = 0, de = 0;
    for (size_t i = 0; i < a.size(); i++)
    {
      nu += (a[i] - ref[i]) * (a[i] - ref[i]);
      de += ref[i] * ref[i];
    }
    return std::sqrt(nu / de);
  };
  double const dense_rel = rel(y_dense, y_host);
  // new per-term coefficients: twice the factors of dimension 0 doubles K x
  for (auto &tv : dterms)
    for (size_t e = 0; e < size_t(nb) * nb * 9; e++)
      tv[e] *= 2.0;
  std::vector<double> ya(N, 0.0), yb(N, 0.0);
  mat.apply<resource::host>(2.0, x.data(), 0.0, ya.data());
  dmat.update_stored_coefficients(dterms);
  dmat.apply<resource::host>(1.0, x.data(), 0.0, yb.data());
  double const dense_update_rel = rel(yb, ya);

  // the multi-call forms: three CSR row blocks, and the GPU pair format in
  // two interleaved chunks
  std::vector<std::vector<int>> lp, li, la;
  int const cuts[4] = {0, int(cells) / 3, 2 * int(cells) / 3, int(cells)};
  for (int c = 0; c < 3; c++)
  {
    std::vector<int> p(1, 0), ix, ia;
    for (int r = cuts[c]; r < cuts[c + 1]; r++)
    {
      for (int j = pntr[r]; j < pntr[r + 1]; j++)
      {
        ix.push_back(col[j]);
        ia.insert(ia.end(), iA.begin() + int64_t(j) * T * d, iA.begin() + int64_t(j + 1) * T * d);
      }
      p.push_back(int(ix.size()));
    }
    lp.push_back(p);
    li.push_back(ix);
    la.push_back(ia);
  }
  kronmult_matrix<double> chunked(d, n, int(cells), int(cells), T, lp, li, la, vA);
  std::vector<std::vector<int>> gr(2), gc(2), ga(2);
  int const ts = mat.tensor_size();
  for (int r = 0; r < int(cells); r++)
    for (int j = pntr[r]; j < pntr[r + 1]; j++)
    {
      gr[j % 2].push_back(r * ts);
      gc[j % 2].push_back(col[j] * ts);
      ga[j % 2].insert(ga[j % 2].end(), iA.begin() + int64_t(j) * T * d,
                       iA.begin() + int64_t(j + 1) * T * d);
    }
  auto paired = kronmult_matrix<double>::from_pair_lists(d, n, int(cells), int(cells), T, gr, gc, ga, vA);
  std::vector<double> y_chunk = y0, y_pairs = y0;
  chunked.apply<resource::host>(0.5, x.data(), -2.0, y_chunk.data());
  paired.apply<resource::host>(0.5, x.data(), -2.0, y_pairs.data());
  double const chunk_rel = rel(y_chunk, y_host), pairs_rel = rel(y_pairs, y_host);

  // caller-owned staging buffers for host applies (set_workspace)
  double *wx = nullptr, *wy = nullptr;
  cudaMalloc(&wx, sizeof(double) * N);
  cudaMalloc(&wy, sizeof(double) * N);
  mat.set_workspace(wx, wy);
  std::vector<double> y_ws = y0, x_staged(N);
  mat.apply<resource::host>(0.5, x.data(), -2.0, y_ws.data());
  cudaMemcpy(x_staged.data(), wx, sizeof(double) * N, cudaMemcpyDeviceToHost);
  double const ws_rel = rel(y_ws, y_host);
  double const ws_used = (x_staged == x) ? 1.0 : 0.0;

  // restart larger than the system must throw std::invalid_argument
  int threw = 0;
  try
  {
    solver::simple_gmres_euler(1e-2, mat, dx, db, N + 1, 1, 1e-12);
  }
  catch (std::invalid_argument const &)
  {
    threw = 1;
  }

  // the 3x3 known answer of the reference solver tests (column-major A)
  std::vector<double> A = {3.383861628748717e+00, 3.210305545769361e+00, 1.723479266939425e+00,
                           1.113343240310116e-02, 3.412141162288144e+00, 1.710451084172946e+00,
                           2.920740795411032e+00, 3.934494120167269e+00, 4.450671104482062e+00};
  std::vector<double> b3 = {2.084406360034887e-01, 6.444769305362776e-01, 3.687335330031937e-01};
  std::vector<double> x3(3, 0.0);
  auto info3 = solver::simple_gmres(A, x3, b3, 3, 3, 2.220446049250313e-16);
  // the same with the reference's point-Jacobi dense preconditioner M
  std::vector<double> M3 = {3.383861628748717e+00, 0.0, 0.0,
                            0.0, 3.412141162288144e+00, 0.0,
                            0.0, 0.0, 4.450671104482062e+00};
  std::vector<double> x3p(3, 0.0);
  auto info3p = solver::simple_gmres(A, x3p, b3, M3, 3, 3, 2.220446049250313e-16);

  // a preconditioner built for another step size is refused
  int dt_threw = 0;
  {
    solver::jacobi_preconditioner pc(mat, 2e-2, ASGK_JACOBI_POINT);
    try
    {
      solver::simple_gmres_euler(1e-2, mat, dx, db, 20, 50, 1e-12, pc);
    }
    catch (std::invalid_argument const &)
    {
      dt_threw = 1;
    }
  }

  // kronmult_matrix<float>: the same operator from FP32 factors, applied
  // on host and device FP32 vectors, and one FP32 implicit step
  double f_host_rel = 1.0, f_dev_rel = 1.0, f_sol_rel = 1.0, f_its = 0.0;
  {
    std::vector<float> vf(vA.begin(), vA.end()), xf(x.begin(), x.end()),
        y0f(y0.begin(), y0.end()), bf(b.begin(), b.end());
    kronmult_matrix<float> fm(d, n, int(cells), int(cells), T, pntr, col, iA, vf);
    std::vector<float> yh = y0f;
    fm.apply<resource::host>(0.5f, xf.data(), -2.0f, yh.data());
    float *fx = nullptr, *fy = nullptr, *fb = nullptr;
    cudaMalloc(&fx, sizeof(float) * N);
    cudaMalloc(&fy, sizeof(float) * N);
    cudaMalloc(&fb, sizeof(float) * N);
    cudaMemcpy(fx, xf.data(), sizeof(float) * N, cudaMemcpyHostToDevice);
    cudaMemcpy(fy, y0f.data(), sizeof(float) * N, cudaMemcpyHostToDevice);
    fm.apply<resource::device>(0.5f, fx, -2.0f, fy);
    std::vector<float> yd(N);
    cudaMemcpy(yd.data(), fy, sizeof(float) * N, cudaMemcpyDeviceToHost);
    cudaMemcpy(fb, bf.data(), sizeof(float) * N, cudaMemcpyHostToDevice);
    cudaMemset(fx, 0, sizeof(float) * N);
    auto fi = solver::simple_gmres_euler(1e-2f, fm, fx, fb, 20, 50, 1e-5f);
    std::vector<float> fs(N);
    cudaMemcpy(fs.data(), fx, sizeof(float) * N, cudaMemcpyDeviceToHost);
    auto relf = [&](std::vector<float> const &a, std::vector<double> const &e) {
      double nu = 0, de = 0;
      for (int64_t i = 0; i < N; i++)
      {
        nu += (double(a[i]) - e[i]) * (double(a[i]) - e[i]);
        de += e[i] * e[i];
      }
      return std::sqrt(nu / de);
    };
    f_host_rel = relf(yh, y_host);
    f_dev_rel  = relf(yd, y_host);
    f_sol_rel  = relf(fs, sol);
    f_its      = fi.iterations;
    cudaFree(fx);
    cudaFree(fy);
    cudaFree(fb);
  }

  std::ofstream o(argv[1], std::ios::binary);
  put(o, pntr);
  put(o, col);
  put(o, iA);
  put(o, vA);
  put(o, x);
  put(o, y0);
  put(o, y_host);
  put(o, y_dev);
  put(o, b);
  put(o, sol);
  put(o, x3);
  put(o, x3p);
  std::vector<double> meta = {double(d), double(n), double(T), double(cells),
                              info.error, double(info.iterations), double(threw),
                              info3.error, double(mat.num_pairs()),
                              double(mat.flops()),
                              double(kronmult_matrix<double>::compute_flops(d, n, T, mat.num_pairs())),
                              global_multi_rel, global_rel,
                              double(mat.num_batch()), double(mat.is_dense()),
                              double(dmat.is_dense()), double(dmat.num_batch()),
                              double(dmat.flops()), dense_rel, dense_update_rel,
                              chunk_rel, pairs_rel, double(chunked.num_pairs()),
                              ws_rel, ws_used, pc_rel, pc_its, pc_err,
                              info3p.error, double(info3p.iterations),
                              double(dt_threw), f_host_rel, f_dev_rel,
                              f_sol_rel, f_its};
  put(o, meta);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(db);
  cudaFree(wx);
  cudaFree(wy);
  std::printf("dropin ok: %d cells, %lld pairs, gmres %d its\n", int(cells),
              (long long)nnz, info.iterations);
  return 0;
}
