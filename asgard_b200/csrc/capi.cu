// C ABI: operator plans, apply entry points and the device-resident GMRES.
#include "gmres_device.cuh"
#include "internal.cuh"
#include "mlp.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <numeric>

namespace asgk
{
std::atomic<int64_t> g_launches{0};
thread_local bool g_recording            = false;
thread_local int64_t g_recorded_launches = 0;
thread_local const double *g_gate        = nullptr;

namespace
{
template<typename T>
int dev_alloc(T **ptr, int64_t count, int64_t &bytes)
{
  *ptr = nullptr;
  if (count <= 0)
    return ASGK_OK;
  size_t const b = size_t(count) * sizeof(T);
  if (cudaMalloc(reinterpret_cast<void **>(ptr), b) != cudaSuccess)
  {
    cudaGetLastError();
    return ASGK_ERR_ALLOC;
  }
  bytes += int64_t(b);
  return ASGK_OK;
}

void free_plan(plan_data &p)
{
  cudaFree(p.row_ptr);
  cudaFree(p.col);
  cudaFree(p.idx);
  cudaFree(p.row_order);
  cudaFree(p.vA64);
  cudaFree(p.vA32);
  if (p.ws_owned)
  {
    cudaFree(p.xw);
    cudaFree(p.yw);
  }
  cudaFree(p.xs);
  cudaFree(p.gptr);
  cudaFree(p.gcol);
  cudaFree(p.gkb);
  cudaFree(p.gB64);
  cudaFree(p.gB32);
  cudaFree(p.slice_row);
  cudaFree(p.slice_len);
  cudaFree(p.slice_beg);
  cudaFree(p.row_slice0);
  cudaFree(p.row_nslice);
  cudaFree(p.gscratch);
  cudaFree(p.gtickets);
  cudaFree(p.gseg);
  cudaFree(p.gcell_order);
  cudaFree(p.gx32);
  cudaFree(p.gjobs);
  cudaFree(p.gchain_last);
  cudaFree(p.gd_ptr);
  cudaFree(p.gd_col);
  cudaFree(p.gd_conn);
  cudaFree(p.gd_rel);
  cudaFree(p.gwork);
  cudaFree(p.vP64);
  cudaFree(p.vP32);
  tc_free(p.tc);
  p = plan_data{};
}

__global__ void k_to_f32(const double *__restrict__ a, float *__restrict__ b,
                         int64_t n)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    b[i] = static_cast<float>(a[i]);
}

// vP[((c*d + k)*T + t)*PAD + e] = vA[c*d*T*9 + (t*d + k)*9 + e] (e < 9), 0 pad
__global__ void k_repack(const double *__restrict__ vA, int64_t nconn, int d,
                         int T, double *__restrict__ v64,
                         float *__restrict__ v32)
{
  int64_t const total = nconn * d * T;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    int64_t const c = i / (d * T);
    int const k     = int((i / T) % d);
    int const t     = int(i % T);
    const double *src = vA + c * d * T * 9 + (t * d + k) * 9;
    for (int e = 0; e < 10; e++)
      v64[i * 10 + e] = (e < 9) ? src[e] : 0.0;
    for (int e = 0; e < 12; e++)
      v32[i * 12 + e] = (e < 9) ? float(src[e]) : 0.0f;
  }
}

// Global mode: finds the dimensions each term acts in (a dimension is
// inactive when its blocks are the identity: I for a self-connection, 0 for
// every other, exactly) and sums each dimension's blocks over the terms
// acting in that dimension alone.  B: [nconn*d][10] (9 values + pad).
// multi: the terms acting in several dimensions, each as (term, its active
// dimensions in increasing order), applied as chains of 1D passes.
int global_blocks(int d, int terms, std::vector<int> const &conn_row,
                  std::vector<int> const &conn_col, const double *vA,
                  std::vector<double> &B, int &n_identity,
                  std::vector<std::vector<int>> &multi)
{
  int64_t const nconn = int64_t(conn_row.size());
  auto blk = [&](int64_t j, int t, int k) {
    return vA + j * d * terms * 9 + int64_t(t * d + k) * 9;
  };
  std::vector<int> active(terms, -1);
  n_identity = 0;
  multi.clear();
  for (int t = 0; t < terms; t++)
  {
    std::vector<int> dims;
    for (int k = 0; k < d; k++)
    {
      bool ident = true;
      for (int64_t j = 0; j < nconn && ident; j++)
      {
        bool const self = conn_row[j] == conn_col[j];
        const double *a = blk(j, t, k);
        for (int e = 0; e < 9 && ident; e++)
          ident = a[e] == ((self && e % 4 == 0) ? 1.0 : 0.0);
      }
      if (!ident)
        dims.push_back(k);
    }
    if (dims.empty())
      ++n_identity;
    else if (dims.size() == 1)
      active[t] = dims[0];
    else
    {
      dims.insert(dims.begin(), t);
      multi.push_back(dims);
    }
  }
  B.assign(size_t(nconn) * d * 10, 0.0);
  for (int t = 0; t < terms; t++)
  {
    int const k = active[t];
    if (k < 0)
      continue;
    for (int64_t j = 0; j < nconn; j++)
      for (int e = 0; e < 9; e++)
        B[(j * d + k) * 10 + e] += blk(j, t, k)[e];
  }
  return ASGK_OK;
}

// The chains of a term acting in m >= 2 dimensions a_0 < ... < a_{m-1}, as
// the reference's permutes (src/device/asgard_kronmult.hpp:152-224) builds
// them: 2^(m-1) chains; in chain c, dimension a_s (s >= 1) takes the lower
// part of its operator when bit s-1 of c is 0, the upper part (diagonal
// included) when 1; a chain applies its upper parts first (in decreasing
// order of s), then the whole operator of a_0, then its lower parts (in
// increasing order of s).  The chains' sum is the term's operator on the
// sparse grid.  Stage entries: (dimension, fill) with fill 0 = upper,
// 1 = both, 2 = lower.
std::vector<std::vector<std::pair<int, int>>> term_chains(std::vector<int> const &dims)
{
  int const m = int(dims.size());
  std::vector<std::vector<std::pair<int, int>>> out;
  for (int c = 0; c < (1 << (m - 1)); c++)
  {
    std::vector<int> signed_dir(m, 0); // -s: upper, +s: lower, 0: both
    for (int s = 1; s < m; s++)
      signed_dir[s] = ((c >> (s - 1)) & 1) ? -s : s;
    std::sort(signed_dir.begin(), signed_dir.end());
    std::vector<std::pair<int, int>> chain;
    for (int v : signed_dir)
      chain.emplace_back(dims[std::abs(v)], v < 0 ? 0 : (v > 0 ? 2 : 1));
    out.push_back(chain);
  }
  return out;
}

int upload_global_blocks(plan_data &p, std::vector<double> const &B)
{
  std::vector<float> B32(B.size() / 10 * 12, 0.0f);
  for (size_t i = 0; i < B.size() / 10; i++)
    for (int e = 0; e < 9; e++)
      B32[i * 12 + e] = float(B[i * 10 + e]);
  ASGK_CUDA(cudaMemcpy(p.gB64, B.data(), sizeof(double) * B.size(),
                       cudaMemcpyHostToDevice));
  ASGK_CUDA(cudaMemcpy(p.gB32, B32.data(), sizeof(float) * B32.size(),
                       cudaMemcpyHostToDevice));
  if (p.tc != nullptr)
    return tc_refresh(p, *p.tc);
  return ASGK_OK;
}

int upload_values(plan_data &p, const double *vA)
{
  ASGK_CUDA(cudaMemcpy(p.vA64, vA, sizeof(double) * p.vA_len,
                       cudaMemcpyHostToDevice));
  if (p.vA_len > 0)
  {
    k_to_f32<<<256, 256>>>(p.vA64, p.vA32, p.vA_len);
    ASGK_LAUNCHED();
  }
  if (p.nconn > 0)
  {
    k_repack<<<256, 256>>>(p.vA64, p.nconn, p.d, p.terms, p.vP64, p.vP32);
    ASGK_LAUNCHED();
  }
  ASGK_CUDA(cudaDeviceSynchronize());
  return ASGK_OK;
}

// Dense-mode factors to the per-connection layout of a conn-mode plan: the
// caller's terms[t] hold, per dimension k, num_1d_blocks^2 column-major n x n
// blocks ordered by (column cell, row cell) (make_kronmult_dense,
// src/asgard_kronmult_matrix.cpp:95-113); connection c = ic*nb + ir keeps
// the d*T blocks of that 1D pair together.
std::vector<double> dense_values(int d, int n, int terms, int nb,
                                 const double *const *tv)
{
  int64_t const nn = int64_t(n) * n;
  int64_t const nc = int64_t(nb) * nb;
  std::vector<double> vA(size_t(nc * d * terms * nn));
  for (int t = 0; t < terms; t++)
    for (int k = 0; k < d; k++)
      for (int64_t c = 0; c < nc; c++)
        std::copy_n(tv[t] + (k * nc + c) * nn, nn,
                    vA.data() + (c * d * terms + t * d + k) * nn);
  return vA;
}

int check_dims(int d, int n, int rows, int cols, int terms)
{
  if (d < 1 || d > 6 || n < 1 || rows < 0 || cols < 0 || terms < 0)
    return ASGK_ERR_INVALID;
  double ts = std::pow(double(n), d);
  if (ts > double(1 << 24))
    return ASGK_ERR_UNSUPPORTED;
  return ASGK_OK;
}

int64_t ipow(int n, int d)
{
  int64_t r = 1;
  for (int i = 0; i < d; i++)
    r *= n;
  return r;
}

// Sets a plan's sizes and allocates its device arrays: CSR pairs with idx_len
// factor indices, the factors (FP64, FP32, repacked per connection for
// n = 3 conn plans) and the staged kernel's x scratch.  Frees what it
// allocated on failure.
int alloc_plan(plan_data &p, int d, int n, int rows, int cols, int terms,
               int64_t nnz, index_mode mode, int64_t vA_len, int64_t idx_len)
{
  int64_t const blk = int64_t(d) * terms * n * n;
  p.d      = d;
  p.n      = n;
  p.rows   = rows;
  p.cols   = cols;
  p.terms  = terms;
  p.tensor = int(ipow(n, d));
  p.nnz    = nnz;
  p.mode   = mode;
  p.vA_len = vA_len;
  if (mode == index_mode::conn && n == 3 && terms > 0)
    p.nconn = vA_len / blk;
  int64_t &B = p.device_bytes;
  int rc     = ASGK_OK;
  if ((rc = dev_alloc(&p.row_ptr, rows + 1, B)) ||
      (rc = dev_alloc(&p.col, std::max<int64_t>(nnz, 1), B)) ||
      (rc = dev_alloc(&p.idx, std::max<int64_t>(idx_len, 1), B)) ||
      (rc = dev_alloc(&p.row_order, std::max(rows, 1), B)) ||
      (rc = dev_alloc(&p.vA64, std::max<int64_t>(vA_len, 1), B)) ||
      (rc = dev_alloc(&p.vA32, std::max<int64_t>(vA_len, 1), B)) ||
      (rc = dev_alloc(&p.vP64, p.nconn * d * terms * 10, B)) ||
      (rc = dev_alloc(&p.vP32, p.nconn * d * terms * 12, B)) ||
      (rc = dev_alloc(&p.xs, terms > 0 ? staged_x_doubles(d, n, cols) : 0, B)))
  {
    free_plan(p);
    return rc;
  }
  return ASGK_OK;
}

// Builds the device plan from host CSR arrays (validated here).
int build_plan(asgk_plan **out, int d, int n, int rows, int cols, int terms,
               std::vector<int64_t> const &row_ptr, const int *col,
               const int *idx, index_mode mode, const double *vA,
               int64_t vA_len)
{
  if (out == nullptr)
    return ASGK_ERR_INVALID;
  *out = nullptr;
  if (int rc = check_dims(d, n, rows, cols, terms))
    return rc;
  if (vA_len < 0 || (vA_len > 0 && vA == nullptr))
    return ASGK_ERR_INVALID;
  int64_t const nnz = row_ptr.empty() ? 0 : row_ptr.back();
  if (row_ptr.size() != size_t(rows) + 1 || row_ptr[0] != 0)
    return ASGK_ERR_INVALID;
  for (int r = 0; r < rows; r++)
    if (row_ptr[r + 1] < row_ptr[r])
      return ASGK_ERR_INVALID;
  if (nnz > 0 && (col == nullptr || (terms > 0 && idx == nullptr)))
    return ASGK_ERR_INVALID;
  for (int64_t i = 0; i < nnz; i++)
    if (col[i] < 0 || col[i] >= cols)
      return ASGK_ERR_INVALID;
  int64_t const nn  = int64_t(n) * n;
  int64_t const blk = int64_t(d) * terms * nn;
  int64_t idx_len   = 0;
  if (terms > 0)
  {
    if (mode == index_mode::expanded)
    {
      idx_len = nnz * terms * d;
      for (int64_t i = 0; i < idx_len; i++)
        if (idx[i] < 0 || int64_t(idx[i]) + nn > vA_len)
          return ASGK_ERR_INVALID;
    }
    else
    {
      idx_len = nnz * d;
      for (int64_t i = 0; i < idx_len; i++)
        if (idx[i] < 0 || (int64_t(idx[i]) + 1) * blk > vA_len)
          return ASGK_ERR_INVALID;
    }
  }
  std::unique_ptr<asgk_plan> plan(new (std::nothrow) asgk_plan());
  if (!plan)
    return ASGK_ERR_ALLOC;
  plan_data &p = plan->p;
  int rc       = alloc_plan(p, d, n, rows, cols, terms, nnz, mode, vA_len, idx_len);
  if (rc)
    return rc;
  // cells by decreasing pair count, ties by index
  std::vector<int> order(rows);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (row_ptr[a + 1] - row_ptr[a]) > (row_ptr[b + 1] - row_ptr[b]);
  });
  auto up = [&](void *dst, const void *src, size_t bytes) -> int {
    if (bytes == 0)
      return ASGK_OK;
    ASGK_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return ASGK_OK;
  };
  // For the staged n = 3, d = 3/4 kernel, each row's pairs are ordered by
  // their factor blocks, the last dimension slowest and dimension 0 fastest:
  // the ten pairs a warp contracts together then mostly share the blocks of
  // dimensions 1..d-1 (read whole) and differ in dimension 0 (read as one
  // column per lane), and a block's reuse distance stays within L1.  The
  // result changes only by the order of the floating-point sums.
  std::vector<int> col_sorted, idx_sorted;
  if (n == 3 && (d == 3 || d == 4) && terms > 0 && nnz > 0)
  {
    int64_t const per = (mode == index_mode::conn) ? d : int64_t(terms) * d;
    col_sorted.resize(nnz);
    idx_sorted.resize(idx_len);
#pragma omp parallel for schedule(dynamic, 16)
    for (int r = 0; r < rows; r++)
    {
      int64_t const b = row_ptr[r], e = row_ptr[r + 1];
      std::vector<int64_t> ord(e - b);
      std::iota(ord.begin(), ord.end(), b);
      std::stable_sort(ord.begin(), ord.end(), [&](int64_t u, int64_t v) {
        for (int k = d - 1; k >= 0; k--)
          if (idx[u * per + k] != idx[v * per + k])
            return idx[u * per + k] < idx[v * per + k];
        return col[u] < col[v];
      });
      for (int64_t i = 0; i < e - b; i++)
      {
        col_sorted[b + i] = col[ord[i]];
        std::copy(idx + ord[i] * per, idx + (ord[i] + 1) * per,
                  idx_sorted.begin() + (b + i) * per);
      }
    }
    col = col_sorted.data();
    idx = idx_sorted.data();
  }
  if ((rc = up(p.row_ptr, row_ptr.data(), sizeof(int64_t) * (rows + 1))) ||
      (rc = up(p.col, col, sizeof(int) * nnz)) ||
      (rc = up(p.idx, idx, sizeof(int) * idx_len)) ||
      (rc = up(p.row_order, order.data(), sizeof(int) * rows)) ||
      (rc = upload_values(p, vA)))
  {
    free_plan(p);
    return rc;
  }
  *out = plan.release();
  return ASGK_OK;
}

cudaStream_t as_stream(asgk_stream s) { return static_cast<cudaStream_t>(s); }

// y = beta*y + alpha*A*x for a dense column-major n x n matrix (one warp per row)
__global__ void k_dense_gemv(int n, const double *__restrict__ A, double alpha,
                             const double *__restrict__ x, double beta,
                             double *__restrict__ y)
{
  int const row  = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int const lane = threadIdx.x & 31;
  if (row >= n)
    return;
  double s = 0;
  for (int j = lane; j < n; j += 32)
    s += A[row + int64_t(j) * n] * x[j];
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0)
    y[row] = (beta == 0.0 ? 0.0 : beta * y[row]) + alpha * s;
}

// FP32 vectors of kronmult_matrix<float> solves to and from the FP64 copies
// the solver works on
__global__ void k_widen(int64_t n, const float *__restrict__ in,
                        double *__restrict__ out)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = double(in[i]);
}
__global__ void k_narrow(int64_t n, const double *__restrict__ in,
                         float *__restrict__ out)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

// ------------------------------------------------------------------ GMRES

// Reference BLAS Givens generation (drotg), as reached by lib_dispatch::rotg.
void rotg(double &a, double &b, double &c, double &s)
{
  double const sa = a, sb = b;
  double const roe   = (std::fabs(sa) > std::fabs(sb)) ? sa : sb;
  double const scale = std::fabs(sa) + std::fabs(sb);
  double r, z;
  if (scale == 0)
  {
    c = 1;
    s = 0;
    r = 0;
    z = 0;
  }
  else
  {
    r = scale * std::sqrt((sa / scale) * (sa / scale) + (sb / scale) * (sb / scale));
    r = (roe >= 0 ? 1.0 : -1.0) * r;
    c = sa / r;
    s = sb / r;
    z = 1;
    if (std::fabs(sa) > std::fabs(sb))
      z = s;
    if (std::fabs(sb) >= std::fabs(sa) && c != 0)
      z = 1 / c;
  }
  a = r;
  b = z;
}

inline void rot(double &x, double &y, double c, double s)
{
  double const tx = c * x + s * y;
  double const ty = c * y - s * x;
  x = tx;
  y = ty;
}

inline int pos_from_indices(int i, int j) { return i + j * (j + 1) / 2; }

// What a recorded GMRES cycle depends on besides the workspace buffers: the
// operator (plan, dt, arithmetic), the preconditioner, the restart length,
// the basis precision of the Gram-Schmidt passes, the Arnoldi steps per
// graph node, whether the preconditioner writes the operator's FP32 input.
struct graph_key
{
  const void *plan = nullptr; // the workspace dies with its plan
  double dt        = 0;
  int precision    = 0;
  uint64_t pc      = 0;       // preconditioner serial (never reused), 0: none
  int restart      = 0;
  bool low_basis   = false;
  int node_steps   = 1;
  bool fused_copy  = false;
  bool operator==(graph_key const &o) const
  {
    return plan == o.plan && dt == o.dt && precision == o.precision &&
           pc == o.pc && restart == o.restart && low_basis == o.low_basis &&
           node_steps == o.node_steps && fused_copy == o.fused_copy;
  }
};

bool g_gmres_graphs     = true; // asgk_set_gmres_graphs
bool g_gmres_low_basis  = true; // asgk_set_gmres_basis
bool g_gmres_fused_copy = true; // asgk_set_gmres_fused_copy
// steps per node of a recorded cycle (asgk_set_gmres_node_steps): at d=4
// level 7 a 138-iteration solve took 9.85 / 8.49 / 8.33 / 8.23 ms with 1 / 4
// / 8 / 16 (node boundaries cost ~10 us, a skipped launch ~1 us)
int g_gmres_node_steps  = 16;
// relative tolerance of the inner solves with the BF16 tensor-core operator
// (asgk_set_bf16_inner_tol): its products carry BF16-rounded operands, so an
// inner solve far below that rounding gains the refinement nothing
double g_bf16_inner_rtol = 1e-3;

// Device workspace of a GMRES solve, kept on the plan between solves.
struct gmres_ws
{
  int64_t N = 0;
  int m = 0;
  bool flexible = false;
  double *V = nullptr, *Z = nullptr, *part = nullptr, *h = nullptr,
         *y = nullptr, *r = nullptr, *e = nullptr;
  double *hh = nullptr; // pinned host mirror of h
  // The solver's scalar reads (norms, Gram-Schmidt sums, the recorded
  // cycle's state) and its write of the least-squares solution go through
  // mapped pinned memory, moved by one-block kernels: a caller streaming
  // large copies on another stream (x out, the next b in) occupies the copy
  // engines, and a small cudaMemcpyAsync would queue behind those copies.
  // Device aliases of hh, hstate and hy (null: mapping unavailable, plain
  // copies instead).
  double *hh_dev = nullptr, *hstate_dev = nullptr;
  double *hy = nullptr, *hy_dev = nullptr; // pinned staging of the LS solution
  // FP32 copy of the basis for the Gram-Schmidt passes of FP32 inner solves
  // (allocated on first use, n * (m + 1))
  float *Vf = nullptr;
  // reduction tickets: [0] update-norm, [1] norm, [2..] multi-dot groups
  unsigned *tickets = nullptr;
  int nblocks = 0;
  // recorded restart cycles (one graph per operator/preconditioner/restart)
  double *dstate = nullptr, *hstate = nullptr; // device state, pinned mirror
  struct cycle_graph
  {
    graph_key key;
    cudaGraph_t graph      = nullptr;
    cudaGraphExec_t exec   = nullptr;
    int kernels_per_step   = 0;
  };
  std::vector<cycle_graph> graphs;
  bool graphs_broken       = false; // a graph call failed: host-driven cycles
  cudaStream_t capture     = nullptr;

  ~gmres_ws() { release(); }
  void drop_graphs()
  {
    for (auto &g : graphs)
    {
      if (g.exec)
        cudaGraphExecDestroy(g.exec);
      if (g.graph)
        cudaGraphDestroy(g.graph);
    }
    graphs.clear();
  }
  void release()
  {
    drop_graphs();
    if (capture)
      cudaStreamDestroy(capture);
    capture = nullptr;
    cudaFree(dstate);
    dstate = nullptr;
    if (hstate)
      cudaFreeHost(hstate);
    hstate     = nullptr;
    hstate_dev = nullptr;
    if (hy)
      cudaFreeHost(hy);
    hy = hy_dev = nullptr;
    cudaFree(V);
    cudaFree(Vf);
    Vf = nullptr;
    cudaFree(Z);
    cudaFree(part);
    cudaFree(h);
    cudaFree(y);
    cudaFree(r);
    cudaFree(e);
    cudaFree(tickets);
    tickets = nullptr;
    if (hh)
      cudaFreeHost(hh);
    V = Z = part = h = y = r = e = hh = hh_dev = nullptr;
    N = 0;
    m = 0;
  }
  int ensure(int64_t n, int restart, bool flex, bool low = false)
  {
    if (n == N && restart <= m && (!flex || Z != nullptr))
    {
      if (!low || Vf != nullptr)
        return ASGK_OK;
      int64_t bytes = 0;
      return dev_alloc(&Vf, n * (m + 1), bytes);
    }
    release();
    int64_t bytes = 0;
    nblocks       = max_reduction_blocks_wide();
    int rc;
    if ((rc = dev_alloc(&V, n * (restart + 1), bytes)) ||
        (flex && (rc = dev_alloc(&Z, n * restart, bytes))) ||
        (low && (rc = dev_alloc(&Vf, n * (restart + 1), bytes))) ||
        (rc = dev_alloc(&part, int64_t(nblocks) * (restart + 2), bytes)) ||
        (rc = dev_alloc(&h, restart + 2, bytes)) ||
        (rc = dev_alloc(&y, restart + 1, bytes)) ||
        (rc = dev_alloc(&r, n, bytes)) || (rc = dev_alloc(&e, n, bytes)) ||
        (rc = dev_alloc(&tickets, 2 + (restart + 2 + 7) / 8, bytes)))
    {
      release();
      return rc;
    }
    if (cudaMemset(tickets, 0, sizeof(unsigned) * (2 + (restart + 2 + 7) / 8)) !=
        cudaSuccess)
    {
      cudaGetLastError();
      release();
      return ASGK_ERR_CUDA;
    }
    if ((rc = dev_alloc(&dstate, state_len(restart), bytes)))
    {
      release();
      return rc;
    }
    if (cudaHostAlloc(reinterpret_cast<void **>(&hh), sizeof(double) * (restart + 2),
                      cudaHostAllocMapped) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void **>(&hstate),
                      sizeof(double) * state_len(restart), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void **>(&hy), sizeof(double) * (restart + 1),
                      cudaHostAllocMapped) != cudaSuccess)
    {
      cudaGetLastError();
      release();
      return ASGK_ERR_ALLOC;
    }
    if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&hh_dev), hh, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&hstate_dev), hstate, 0) !=
            cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&hy_dev), hy, 0) != cudaSuccess)
    {
      cudaGetLastError();
      hh_dev = hstate_dev = hy_dev = nullptr;
    }
    N        = n;
    m        = restart;
    flexible = flex;
    return ASGK_OK;
  }
};

// operator and preconditioner callbacks take the stream they launch on (the
// solve's stream, or the capture stream while a cycle graph is recorded)
using matvec_t  = std::function<int(double alpha, const double *x, double beta,
                                    double *y, cudaStream_t s)>;
// (with scale_state, v *= scale_state[1] in place first: a recorded step's
// normalisation of its basis vector, fused into the preconditioner; with
// vcopy, also vcopy = FP32(v): the basis copy of an FP32 inner solve)
using precond_t = std::function<int(double *v, double *z,
                                    const double *scale_state, float *vcopy,
                                    cudaStream_t s)>;

struct core_stats
{
  int total   = 0; // reference iteration count
  int matvecs = 0;
  int pcalls  = 0;
  int restarts = 0;
  double err  = 0;
  int status  = ASGK_OK;
  bool verified = false;  // stopped on a recomputed residual
  bool stagnated = false; // a preconditioned cycle reduced the residual < 10%
};

// start of a recorded cycle: the residual estimate, g[0] and the tolerance
__global__ void k_cycle_start(double *st, double inner_res, double tol)
{
  if (blockIdx.x == 0 && threadIdx.x == 0)
  {
    st[0]          = inner_res;
    st[1]          = 1.0;
    st[2]          = 0.0;
    st[3]          = 0.0;
    st[4]          = ASGK_OK;
    st[5]          = tol;
    st[kGoSlot]    = 1.0;
    st[kStateHead] = inner_res;
  }
}

// dst[0..n) = src[0..n): one block, for the few values the solver moves
// between device memory and mapped pinned host memory
__global__ void k_move_small(double *__restrict__ dst, const double *__restrict__ src,
                             int n)
{
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    dst[i] = src[i];
}

// host = src[0..n) (read after the next synchronisation of s): through the
// mapped alias when there is one, else a copy
int read_small(double *host, double *host_dev, const double *src, int n,
               cudaStream_t s)
{
  if (host_dev != nullptr)
  {
    k_move_small<<<1, 64, 0, s>>>(host_dev, src, n);
    ASGK_LAUNCHED();
    return ASGK_OK;
  }
  ASGK_CUDA(cudaMemcpyAsync(host, src, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  return ASGK_OK;
}

int norm2(gmres_ws &ws, const double *v, int64_t n, double &out,
          cudaStream_t s)
{
  if (int rc = launch_norm2_h(v, n, ws.part, ws.tickets + 1, ws.h, s))
    return rc;
  if (int rc = read_small(ws.hh, ws.hh_dev, ws.h, 1, s))
    return rc;
  ASGK_CUDA(cudaStreamSynchronize(s));
  out = std::sqrt(ws.hh[0]);
  return ASGK_OK;
}

// Records one restart cycle: a chain of conditional nodes of S =
// key.node_steps Arnoldi steps each, the basis columns of every step fixed at
// record time (preconditioner, operator, the two Gram-Schmidt passes, the
// second ending in the Givens step, and the scaling of the new basis vector:
// folded into the next step's preconditioner when there is one, or with an
// FP32 basis copy (low) a kernel that scales and writes the copy).  Node 0
// always runs; the Givens step that ends node b opens node b + 1 only while
// the cycle goes on, so a cycle runs with no host round trip and stops where
// the host-driven loop would.  With S > 1 the kernels of each step read the
// go flag the previous step's Givens update left and return at once when the
// cycle has stopped inside the node: a node boundary costs far more than an
// empty launch.
int record_cycle(gmres_ws &ws, int64_t n, matvec_t const &mat,
                 precond_t const *pc, int restart, gmres_ws::cycle_graph &out)
{
  if (!ws.capture &&
      cudaStreamCreateWithFlags(&ws.capture, cudaStreamNonBlocking) != cudaSuccess)
    return ASGK_ERR_CUDA;
  cudaStream_t const cs = ws.capture;
  bool const low        = out.key.low_basis;
  int const S           = std::max(1, std::min(out.key.node_steps, restart));
  int const nodes       = (restart + S - 1) / S;
  cudaGraph_t graph     = nullptr;
  if (cudaGraphCreate(&graph, 0) != cudaSuccess)
    return ASGK_ERR_CUDA;
  g_recording         = true;
  g_recorded_launches = 0;
  g_gate              = nullptr;
  std::vector<cudaGraphConditionalHandle> hs(nodes);
  int rc = ASGK_OK;
  for (int b = 0; b < nodes && rc == ASGK_OK; b++)
    if (cudaGraphConditionalHandleCreate(&hs[b], graph, b == 0 ? 1u : 0u,
                                         cudaGraphCondAssignDefault) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
  cudaGraphNode_t prev = nullptr;
  int kps              = 0;
  for (int b = 0; b < nodes && rc == ASGK_OK; b++)
  {
    cudaGraphNodeParams np{};
    np.type                = cudaGraphNodeTypeConditional;
    np.conditional.handle  = hs[b];
    np.conditional.type    = cudaGraphCondTypeIf;
    np.conditional.size    = 1;
    cudaGraphNode_t node   = nullptr;
    if (cudaGraphAddNode(&node, graph, prev ? &prev : nullptr, prev ? 1 : 0, &np) !=
        cudaSuccess)
    {
      rc = ASGK_ERR_CUDA;
      break;
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed) != cudaSuccess)
    {
      rc = ASGK_ERR_CUDA;
      break;
    }
    int const i_end = std::min(restart, (b + 1) * S);
    for (int i = b * S; i < i_end && rc == ASGK_OK; i++)
    {
      // the first step of a node runs whenever the node does
      g_gate               = (S > 1 && i > b * S) ? ws.dstate + kGoSlot : nullptr;
      int64_t const before = g_recorded_launches;
      double *vi  = ws.V + int64_t(i) * n;
      double *w   = ws.V + int64_t(i + 1) * n;
      int const k = i + 1;
      if (pc)
      {
        // the preconditioner also normalises v_i (step i-1 left 1/||w|| in
        // the state; v_0 was normalised before the cycle) and writes its FP32
        // copy
        double *zi = ws.Z + int64_t(i) * n;
        rc         = (*pc)(vi, zi, i > 0 ? ws.dstate : nullptr,
                           (i > 0 && low) ? ws.Vf + int64_t(i) * n : nullptr, cs);
        if (rc == ASGK_OK)
          rc = mat(1.0, zi, 0.0, w, cs);
      }
      else
        rc = mat(1.0, vi, 0.0, w, cs);
      if (rc == ASGK_OK)
        rc = low ? launch_multidot_hf(ws.Vf, n, k, w, n, ws.part, ws.tickets + 2, ws.h, cs)
                 : launch_multidot_h(ws.V, n, k, w, n, ws.part, ws.tickets + 2, ws.h, cs);
      if (rc == ASGK_OK)
      {
        givens_args ga;
        ga.state    = ws.dstate;
        ga.step     = i;
        ga.restart  = restart;
        ga.has_next = (i + 1 == i_end && b + 1 < nodes) ? 1 : 0;
        ga.next     = ga.has_next ? hs[b + 1] : hs[b];
        rc = low ? launch_update_norm_hf(ws.Vf, n, k, ws.h, w, n, ws.part, ws.tickets,
                                         ws.h + k, cs, &ga)
                 : launch_update_norm_h(ws.V, n, k, ws.h, w, n, ws.part, ws.tickets,
                                        ws.h + k, cs, &ga);
      }
      // without a preconditioner to fold it into, w is normalised here, with
      // its FP32 copy when there is one.  The last step's w is never read
      // (the solution update uses v_0..v_{k-1}), so with S > 1 this kernel
      // reads the go flag this step's Givens update just wrote.
      if (rc == ASGK_OK && !pc)
      {
        g_gate = (S > 1) ? ws.dstate + kGoSlot : nullptr;
        rc = low ? launch_store_basis(w, ws.Vf + int64_t(i + 1) * n, n, ws.dstate, 0.0, cs)
                 : launch_scale_by(w, n, ws.dstate, cs);
      }
      if (i == 0)
        kps = int(g_recorded_launches - before);
    }
    g_gate = nullptr;
    cudaGraph_t captured = nullptr;
    if (cudaStreamEndCapture(cs, &captured) != cudaSuccess && rc == ASGK_OK)
      rc = ASGK_ERR_CUDA;
    prev = node;
  }
  // what was launched while recording runs later, counted per executed step
  g_recording = false;
  g_gate      = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (rc == ASGK_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
    rc = ASGK_ERR_CUDA;
  if (rc != ASGK_OK)
  {
    cudaGetLastError();
    cudaGraphDestroy(graph);
    return rc;
  }
  out.graph            = graph;
  out.exec             = exec;
  out.kernels_per_step = kps;
  return ASGK_OK;
}

// The recorded cycle for this operator/preconditioner/restart (recorded on
// first use, up to four kept), or null: recording is off or failed once.
gmres_ws::cycle_graph const *cycle_graph_for(gmres_ws &ws, int64_t n,
                                             matvec_t const &mat,
                                             precond_t const *pc, int restart,
                                             graph_key const &key)
{
  if (ws.graphs_broken || !g_gmres_graphs)
    return nullptr;
  for (auto &g : ws.graphs)
    if (g.key == key)
      return &g;
  if (ws.graphs.size() >= 4)
  {
    auto &old = ws.graphs.front();
    cudaGraphExecDestroy(old.exec);
    cudaGraphDestroy(old.graph);
    ws.graphs.erase(ws.graphs.begin());
  }
  gmres_ws::cycle_graph cg;
  cg.key = key;
  if (record_cycle(ws, n, mat, pc, restart, cg) != ASGK_OK)
  {
    std::fprintf(stderr, "asgard_b200: recording a GMRES cycle failed; "
                         "cycles are driven from the host\n");
    ws.graphs_broken = true;
    return nullptr;
  }
  ws.graphs.push_back(cg);
  return &ws.graphs.back();
}

// solver::simple_gmres (src/solver.cpp:157-298) on device vectors.  With a
// preconditioner it is the flexible (right-preconditioned) variant: z_j =
// M(v_j) is stored and the update is x += Z y, so the estimated residual is
// that of the unpreconditioned system.  As in the reference, the last Givens
// rotation is not applied to the right-hand side once the tolerance is met.
//
// verify: the estimate is not trusted -- a cycle that meets the tolerance by
// its estimate is followed by the restart residual r = b - A x, and the solve
// stops only when ||r|| meets the tolerance (the relative-tolerance mode,
// whose contract is the true residual).
int gmres_core(gmres_ws &ws, int64_t n, matvec_t const &mat,
               precond_t const *pc, double *x, const double *b, int restart,
               int max_outer, double tol, core_stats &st, cudaStream_t s,
               bool verify = false, graph_key const *gk = nullptr,
               bool low_basis = false)
{
  bool const flex = (pc != nullptr);
  bool const low  = (gk != nullptr) ? gk->low_basis : low_basis;
  if (int rc = ws.ensure(n, restart, flex, low))
    return rc;
  std::vector<double> proj(size_t(restart) * (restart + 1) / 2, 0.0);
  std::vector<double> sines(restart + 1, 0.0), cosines(restart + 1, 0.0),
      ksol(restart + 1, 0.0);
  int outer       = 0;
  double inner_res = 0, outer_res = tol + 1, cycle_start = -1;
  while (outer_res > tol && outer < max_outer)
  {
    double *r0 = ws.V;
    if (int rc = launch_copy(r0, b, n, s))
      return rc;
    if (int rc = mat(-1.0, x, 1.0, r0, s))
      return rc;
    ++st.total;
    ++st.matvecs;
    if (int rc = norm2(ws, r0, n, inner_res, s))
      return rc;
    if (!std::isfinite(inner_res))
    {
      st.status = ASGK_ERR_NONFINITE;
      st.err    = inner_res;
      return ASGK_OK;
    }
    if (inner_res == 0.0 || (verify && inner_res <= tol))
    {
      outer_res = inner_res;
      st.verified = true;
      break;
    }
    if (flex && cycle_start >= 0 && inner_res > 0.9 * cycle_start)
    {
      // the preconditioned cycle did not reduce the residual by 10%
      st.stagnated = true;
      outer_res    = inner_res;
      break;
    }
    cycle_start = inner_res;
    if (int rc = low ? launch_store_basis(r0, ws.Vf, n, nullptr, 1.0 / inner_res, s)
                     : launch_scale(r0, n, 1.0 / inner_res, s))
      return rc;
    ksol[0] = inner_res;
    int inner = 0;
    gmres_ws::cycle_graph const *cg =
        (gk != nullptr && inner_res > tol)
            ? cycle_graph_for(ws, n, mat, pc, restart, *gk)
            : nullptr;
    if (cg != nullptr)
    {
      // the recorded cycle: one launch, one read of its state
      k_cycle_start<<<1, 32, 0, s>>>(ws.dstate, inner_res, tol);
      ASGK_LAUNCHED();
      ASGK_CUDA(cudaGraphLaunch(cg->exec, s));
      if (int rc = read_small(ws.hstate, ws.hstate_dev, ws.dstate, state_len(restart), s))
        return rc;
      ASGK_CUDA(cudaStreamSynchronize(s));
      const double *hs = ws.hstate;
      inner            = int(hs[3]);
      count_launch(int64_t(inner) * cg->kernels_per_step);
      st.total += inner;
      st.matvecs += inner;
      if (flex)
        st.pcalls += inner;
      if (int(hs[4]) == ASGK_ERR_NONFINITE)
      {
        st.status = ASGK_ERR_NONFINITE;
        st.err    = hs[2];
        return ASGK_OK;
      }
      inner_res         = hs[0];
      const double *g   = hs + kStateHead;
      const double *Hp  = g + 3 * int64_t(restart + 1);
      std::copy(g, g + inner, ksol.begin());
      std::copy(Hp, Hp + int64_t(inner) * (inner + 1) / 2, proj.begin());
    }
    while (cg == nullptr && inner_res > tol && inner < restart)
    {
      double *vi = ws.V + int64_t(inner) * n;
      double *w  = ws.V + int64_t(inner + 1) * n;
      if (flex)
      {
        double *zi = ws.Z + int64_t(inner) * n;
        if (int rc = (*pc)(vi, zi, nullptr, nullptr, s))
          return rc;
        ++st.pcalls;
        if (int rc = mat(1.0, zi, 0.0, w, s))
          return rc;
      }
      else if (int rc = mat(1.0, vi, 0.0, w, s))
        return rc;
      ++st.total;
      ++st.matvecs;
      int const k = inner + 1;
      if (int rc = low ? launch_multidot_hf(ws.Vf, n, k, w, n, ws.part,
                                            ws.tickets + 2, ws.h, s)
                       : launch_multidot_h(ws.V, n, k, w, n, ws.part,
                                           ws.tickets + 2, ws.h, s))
        return rc;
      if (int rc = low ? launch_update_norm_hf(ws.Vf, n, k, ws.h, w, n, ws.part,
                                               ws.tickets, ws.h + k, s)
                       : launch_update_norm_h(ws.V, n, k, ws.h, w, n, ws.part,
                                              ws.tickets, ws.h + k, s))
        return rc;
      if (int rc = read_small(ws.hh, ws.hh_dev, ws.h, k + 1, s))
        return rc;
      ASGK_CUDA(cudaStreamSynchronize(s));
      double const nrm = std::sqrt(ws.hh[k]);
      if (!std::isfinite(nrm))
      {
        st.status = ASGK_ERR_NONFINITE;
        st.err    = nrm;
        return ASGK_OK;
      }
      if (nrm > 0)
        if (int rc = low ? launch_store_basis(w, ws.Vf + int64_t(inner + 1) * n, n,
                                              nullptr, 1.0 / nrm, s)
                         : launch_scale(w, n, 1.0 / nrm, s))
          return rc;
      double *coeffs = proj.data() + pos_from_indices(0, inner);
      for (int j = 0; j < k; j++)
        coeffs[j] = ws.hh[j];
      for (int j = 0; j < inner; j++)
        rot(coeffs[j], coeffs[j + 1], cosines[j], sines[j]);
      double beta = nrm;
      rotg(coeffs[inner], beta, cosines[inner], sines[inner]);
      inner_res = std::fabs(sines[inner] * ksol[inner]);
      if (inner_res > tol && inner < restart)
      {
        ksol[inner + 1] = 0.0;
        rot(ksol[inner], ksol[inner + 1], cosines[inner], sines[inner]);
      }
      ++inner;
      if (nrm == 0.0) // exact solution inside the Krylov space
        break;
    }
    if (inner > 0)
    {
      // tpsv: upper, no transpose, non-unit, packed column-major
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
      std::memcpy(ws.hy, ksol.data(), sizeof(double) * inner);
      if (ws.hy_dev != nullptr)
      {
        k_move_small<<<1, 64, 0, s>>>(ws.y, ws.hy_dev, inner);
        ASGK_LAUNCHED();
      }
      else
        ASGK_CUDA(cudaMemcpyAsync(ws.y, ws.hy, sizeof(double) * inner,
                                  cudaMemcpyHostToDevice, s));
      if (int rc = launch_gemv_add(flex ? ws.Z : ws.V, n, inner, ws.y, x, n, s))
        return rc;
      // ksol is read by the copy above before it is reused
      ASGK_CUDA(cudaStreamSynchronize(s));
    }
    ++outer;
    ++st.restarts;
    outer_res = inner_res;
    if (verify && outer_res <= tol)
      outer_res = tol + 1; // confirm on the restart residual
  }
  if (verify && !st.verified && outer >= max_outer)
    outer_res = inner_res;
  st.err = outer_res;
  if (outer_res > tol)
    st.status = ASGK_ERR_NOT_CONVERGED;
  return ASGK_OK;
}

} // namespace
} // namespace asgk

// Workspace lives beside the plan (kept out of plan_data so the kernels'
// view of the plan stays trivially copyable).
namespace
{
struct plan_extras
{
  asgk::gmres_ws ws;
};
std::vector<std::pair<asgk_plan *, plan_extras *>> g_extras;

plan_extras *extras_of(asgk_plan *p, bool create)
{
  for (auto &e : g_extras)
    if (e.first == p)
      return e.second;
  if (!create)
    return nullptr;
  auto *x = new plan_extras();
  g_extras.emplace_back(p, x);
  return x;
}

void drop_extras(asgk_plan *p)
{
  for (size_t i = 0; i < g_extras.size(); i++)
    if (g_extras[i].first == p)
    {
      delete g_extras[i].second;
      g_extras.erase(g_extras.begin() + i);
      return;
    }
}
} // namespace

using namespace asgk;

extern "C"
{
const char *asgk_status_string(int status)
{
  switch (status)
  {
  case ASGK_OK: return "success";
  case ASGK_ERR_INVALID: return "invalid argument";
  case ASGK_ERR_UNSUPPORTED: return "unsupported dimension or size";
  case ASGK_ERR_CUDA: return "CUDA runtime error";
  case ASGK_ERR_ALLOC: return "allocation failed";
  case ASGK_ERR_BREAKDOWN: return "GMRES breakdown";
  case ASGK_ERR_NOT_CONVERGED: return "GMRES did not converge";
  case ASGK_ERR_NONFINITE: return "non-finite residual";
  case ASGK_ERR_NOALLOC_LIMIT:
    return "size exceeds the fixed scratch of the allocation-free entry point";
  case ASGK_ERR_DEVICE_TIMEOUT:
    return "a kernel's bounded wait on its shared-memory copies expired";
  default: return "unknown status";
  }
}

int64_t asgk_launch_count(void) { return g_launches.load(); }

int asgk_device_status(int reset)
{
  try
  {
    int code = ASGK_OK;
    ASGK_CUDA(cudaDeviceSynchronize());
    if (int rc = read_device_error(reset, &code))
      return rc;
    return code;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_device_info(int *sm_count, int *cc_major, int *cc_minor)
{
  try
  {
    int dev = 0;
    ASGK_CUDA(cudaGetDevice(&dev));
    if (sm_count)
      ASGK_CUDA(cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev));
    if (cc_major)
      ASGK_CUDA(cudaDeviceGetAttribute(cc_major, cudaDevAttrComputeCapabilityMajor, dev));
    if (cc_minor)
      ASGK_CUDA(cudaDeviceGetAttribute(cc_minor, cudaDevAttrComputeCapabilityMinor, dev));
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_create(asgk_plan **plan, int d, int n, int num_rows,
                     int num_cols, int num_terms, const int64_t *row_ptr,
                     const int *col_indx, const int *iA, const double *vA,
                     int64_t vA_len)
{
  try
  {
    if (row_ptr == nullptr || num_rows < 0)
      return ASGK_ERR_INVALID;
    std::vector<int64_t> rp(row_ptr, row_ptr + num_rows + 1);
    return build_plan(plan, d, n, num_rows, num_cols, num_terms, rp, col_indx,
                      iA, index_mode::expanded, vA, vA_len);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_create_conn(asgk_plan **plan, int d, int n, int num_rows,
                          int num_cols, int num_terms, const int64_t *row_ptr,
                          const int *col_indx, const int *conn,
                          const double *vA, int64_t vA_len)
{
  try
  {
    if (row_ptr == nullptr || num_rows < 0)
      return ASGK_ERR_INVALID;
    std::vector<int64_t> rp(row_ptr, row_ptr + num_rows + 1);
    return build_plan(plan, d, n, num_rows, num_cols, num_terms, rp, col_indx,
                      conn, index_mode::conn, vA, vA_len);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_create_pairs(asgk_plan **plan, int d, int n, int num_rows,
                           int num_cols, int num_terms, int64_t num_batch,
                           const int *iy, const int *ix, const int *iA,
                           const double *vA, int64_t vA_len)
{
  try
  {
    if (plan == nullptr)
      return ASGK_ERR_INVALID;
    if (int rc = check_dims(d, n, num_rows, num_cols, num_terms))
      return rc;
    if (num_batch < 0 || (num_batch > 0 && (iy == nullptr || ix == nullptr)))
      return ASGK_ERR_INVALID;
    int64_t const ts = ipow(n, d);
    std::vector<int64_t> rp(num_rows + 1, 0);
    for (int64_t i = 0; i < num_batch; i++)
    {
      if (iy[i] < 0 || iy[i] % ts != 0 || iy[i] / ts >= num_rows ||
          ix[i] < 0 || ix[i] % ts != 0 || ix[i] / ts >= num_cols)
        return ASGK_ERR_INVALID;
      rp[iy[i] / ts + 1]++;
    }
    for (int r = 0; r < num_rows; r++)
      rp[r + 1] += rp[r];
    std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
    std::vector<int> col(num_batch);
    int64_t const per = int64_t(num_terms) * d;
    std::vector<int> ia(num_batch * per);
    for (int64_t i = 0; i < num_batch; i++)
    {
      int64_t const dst = fill[iy[i] / ts]++;
      col[dst]          = int(ix[i] / ts);
      if (per > 0)
        std::copy_n(iA + i * per, per, ia.data() + dst * per);
    }
    return build_plan(plan, d, n, num_rows, num_cols, num_terms, rp, col.data(),
                      ia.data(), index_mode::expanded, vA, vA_len);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_create_dense(asgk_plan **plan, int d, int n, int num_rows,
                           int num_cols, int num_terms,
                           const double *const *terms, const int *elem,
                           int64_t elem_len, int row_offset, int col_offset,
                           int num_1d_blocks)
{
  try
  {
    if (plan == nullptr)
      return ASGK_ERR_INVALID;
    *plan = nullptr;
    if (int rc = check_dims(d, n, num_rows, num_cols, num_terms))
      return rc;
    if (row_offset < 0 || col_offset < 0)
      return ASGK_ERR_INVALID;
    int64_t const npairs = (num_terms > 0) ? int64_t(num_rows) * num_cols : 0;
    int const nb         = (num_terms > 0) ? num_1d_blocks : 0;
    if (num_terms > 0)
    {
      if (terms == nullptr || num_1d_blocks < 1 ||
          int64_t(num_1d_blocks) * num_1d_blocks > (int64_t(1) << 30))
        return ASGK_ERR_INVALID;
      for (int t = 0; t < num_terms; t++)
        if (terms[t] == nullptr)
          return ASGK_ERR_INVALID;
    }
    if (npairs > 0)
    {
      int64_t const need =
          int64_t(d) * std::max(int64_t(row_offset) + num_rows,
                                int64_t(col_offset) + num_cols);
      if (elem == nullptr || elem_len < need)
        return ASGK_ERR_INVALID;
      for (int64_t i = 0; i < need; i++)
        if (elem[i] < 0 || elem[i] >= nb)
          return ASGK_ERR_INVALID;
    }
    // every (row, col) pair, columns in order; per pair the d connections
    // elem_col[k]*nb + elem_row[k]
    std::vector<int64_t> rp(size_t(num_rows) + 1);
    for (int r = 0; r <= num_rows; r++)
      rp[r] = (npairs > 0) ? int64_t(r) * num_cols : 0;
    std::vector<int> col(static_cast<size_t>(npairs));
    std::vector<int> conn(static_cast<size_t>(npairs) * d);
  #pragma omp parallel for schedule(static)
    for (int r = 0; r < (npairs > 0 ? num_rows : 0); r++)
    {
      const int *er = elem + int64_t(r + row_offset) * d;
      for (int c = 0; c < num_cols; c++)
      {
        int64_t const p = int64_t(r) * num_cols + c;
        const int *ec   = elem + int64_t(c + col_offset) * d;
        col[p]          = c;
        for (int k = 0; k < d; k++)
          conn[p * d + k] = ec[k] * nb + er[k];
      }
    }
    std::vector<double> vA;
    if (num_terms > 0)
      vA = dense_values(d, n, num_terms, nb, terms);
    if (int rc = build_plan(plan, d, n, num_rows, num_cols, num_terms, rp,
                            col.data(), conn.data(), index_mode::conn,
                            vA.data(), int64_t(vA.size())))
      return rc;
    (*plan)->p.dense    = true;
    (*plan)->p.dense_nb = nb;
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_set_workspace(asgk_plan *plan, double *x, int64_t x_len,
                            double *y, int64_t y_len)
{
  try
  {
    if (!plan || !x || !y)
      return ASGK_ERR_INVALID;
    auto &p = plan->p;
    if (x_len < int64_t(p.cols) * p.tensor || y_len < int64_t(p.rows) * p.tensor)
      return ASGK_ERR_INVALID;
    if (p.ws_owned && p.xw)
    {
      ASGK_CUDA(cudaDeviceSynchronize()); // an apply_host may still use them
      cudaFree(p.xw);
      cudaFree(p.yw);
      p.device_bytes -= sizeof(double) * (std::max<int64_t>(int64_t(p.cols) * p.tensor, 1) +
                                          std::max<int64_t>(int64_t(p.rows) * p.tensor, 1));
    }
    p.xw       = x;
    p.yw       = y;
    p.ws_owned = false;
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_create_grid(asgk_plan **plan, int d, int n, int level,
                          int num_terms, const double *vA, int64_t vA_len)
{
  try
  {
    if (plan == nullptr)
      return ASGK_ERR_INVALID;
    *plan = nullptr;
    if (d < 1 || d > 6 || level < 0 || level > 12 || num_terms < 0 ||
        (num_terms > 0 && vA == nullptr))
      return ASGK_ERR_INVALID;
    if (int rc = check_dims(d, n, 0, 0, num_terms))
      return rc;
    int64_t const ncells = asgk_sparse_grid(d, level, nullptr);
    if (ncells <= 0 || ncells > (int64_t(1) << 30))
      return ASGK_ERR_UNSUPPORTED;
    int const cells = int(ncells);
    std::vector<int> table(size_t(cells) * 2 * d);
    asgk_sparse_grid(d, level, table.data());
    int R = 0, nconn = 0;
    if (int rc = asgk_connect_1d(level, &R, &nconn, nullptr, nullptr))
      return rc;
    std::vector<int> pntr(R + 1), indx(nconn);
    asgk_connect_1d(level, &R, &nconn, pntr.data(), indx.data());
    int64_t const blk = int64_t(d) * num_terms * n * n;
    if (vA_len != int64_t(nconn) * blk)
      return ASGK_ERR_INVALID;
    std::vector<int> lut(size_t(R) * R, -1), oned(size_t(cells) * d);
    for (int r = 0; r < R; r++)
      for (int j = pntr[r]; j < pntr[r + 1]; j++)
        lut[size_t(r) * R + indx[j]] = j;
    for (int c = 0; c < cells; c++)
      for (int k = 0; k < d; k++)
      {
        int const lv = table[size_t(c) * 2 * d + k], ps = table[size_t(c) * 2 * d + d + k];
        oned[size_t(c) * d + k] = (lv == 0) ? 0 : (1 << (lv - 1)) + ps;
      }
    // candidates in the order each row's pairs are kept: the staged n = 3,
    // d = 3/4 kernel wants them by factor blocks, last dimension slowest (the
    // order build_plan sorts host lists into); table order otherwise
    std::vector<int> cand(cells);
    std::iota(cand.begin(), cand.end(), 0);
    if (n == 3 && (d == 3 || d == 4) && num_terms > 0)
      std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) {
        for (int k = d - 1; k >= 0; k--)
          if (oned[size_t(a) * d + k] != oned[size_t(b) * d + k])
            return oned[size_t(a) * d + k] < oned[size_t(b) * d + k];
        return a < b;
      });
    int *d_oned = nullptr, *d_cand = nullptr, *d_lut = nullptr;
    int64_t *d_counts = nullptr;
    int64_t scratch   = 0;
    auto release = [&]() {
      cudaFree(d_oned);
      cudaFree(d_cand);
      cudaFree(d_lut);
      cudaFree(d_counts);
    };
    int rc = ASGK_OK;
    if ((rc = dev_alloc(&d_oned, int64_t(oned.size()), scratch)) ||
        (rc = dev_alloc(&d_cand, cells, scratch)) ||
        (rc = dev_alloc(&d_lut, int64_t(lut.size()), scratch)) ||
        (rc = dev_alloc(&d_counts, cells, scratch)))
    {
      release();
      return rc;
    }
    std::vector<int64_t> counts(cells), row_ptr(size_t(cells) + 1, 0);
    if (cudaMemcpy(d_oned, oned.data(), sizeof(int) * oned.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(d_cand, cand.data(), sizeof(int) * cand.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(d_lut, lut.data(), sizeof(int) * lut.size(), cudaMemcpyHostToDevice))
      rc = ASGK_ERR_CUDA;
    if (!rc)
      rc = launch_count_pairs(d, cells, d_oned, d_cand, d_lut, R, d_counts, nullptr);
    if (!rc && cudaMemcpy(counts.data(), d_counts, sizeof(int64_t) * cells,
                          cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
    if (rc)
    {
      release();
      return rc;
    }
    for (int r = 0; r < cells; r++)
      row_ptr[r + 1] = row_ptr[r] + counts[r];
    int64_t const nnz = row_ptr[cells];
    std::unique_ptr<asgk_plan> pl(new (std::nothrow) asgk_plan());
    if (!pl)
    {
      release();
      return ASGK_ERR_ALLOC;
    }
    plan_data &p = pl->p;
    // every pair carries its d connection indices (written by the fill)
    if ((rc = alloc_plan(p, d, n, cells, cells, num_terms, nnz, index_mode::conn,
                         vA_len, nnz * d)))
    {
      release();
      return rc;
    }
    std::vector<int> order(cells);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return counts[a] > counts[b]; });
    if (cudaMemcpy(p.row_ptr, row_ptr.data(), sizeof(int64_t) * row_ptr.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p.row_order, order.data(), sizeof(int) * order.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
    if (!rc && nnz > 0)
      rc = launch_fill_pairs(d, cells, d_oned, d_cand, d_lut, R, p.row_ptr, p.col,
                             p.idx, nullptr);
    if (!rc)
      rc = upload_values(p, vA);
    release();
    if (rc)
    {
      free_plan(p);
      return rc;
    }
    *plan = pl.release();
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_kind(const asgk_plan *plan)
{
  if (!plan)
    return -ASGK_ERR_INVALID;
  return plan->p.global ? 2 : (plan->p.dense ? 1 : 0);
}

int asgk_plan_update_terms(asgk_plan *plan, const double *const *terms,
                           int num_terms)
{
  try
  {
    if (!plan || !plan->p.dense || num_terms != plan->p.terms ||
        (num_terms > 0 && terms == nullptr))
      return ASGK_ERR_INVALID;
    for (int t = 0; t < num_terms; t++)
      if (terms[t] == nullptr)
        return ASGK_ERR_INVALID;
    auto &p = plan->p;
    if (num_terms == 0)
      return ASGK_OK;
    std::vector<double> vA = dense_values(p.d, p.n, p.terms, p.dense_nb, terms);
    return upload_values(p, vA.data());
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

void asgk_plan_destroy(asgk_plan *plan)
{
  if (!plan)
    return;
  drop_extras(plan);
  free_plan(plan->p);
  delete plan;
}

int asgk_plan_update_values(asgk_plan *plan, const double *vA, int64_t vA_len)
{
  try
  {
    if (!plan || plan->p.dense || vA_len != plan->p.vA_len || (vA_len > 0 && !vA))
      return ASGK_ERR_INVALID;
    auto &p = plan->p;
    if (p.global)
    {
      std::vector<double> B;
      int n_identity = 0;
      std::vector<std::vector<int>> multi;
      if (int rc = global_blocks(p.d, p.terms, p.g_conn_row, p.g_conn_col, vA, B,
                                 n_identity, multi))
        return rc;
      // the chains are built for the dimensions each term acts in
      if (multi != p.g_multi)
        return ASGK_ERR_INVALID;
      if (int rc = upload_global_blocks(p, B))
        return rc;
      // the identity terms enter the launches as a scalar, which recorded
      // GMRES cycles hold: a change of their count drops the recordings
      if (p.g_identity != n_identity)
        if (auto *ex = extras_of(plan, false))
          ex->ws.drop_graphs();
      p.g_identity = n_identity;
    }
    return upload_values(p, vA);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_create_global(asgk_plan **plan, int d, int n, int level,
                            int num_cells, const int *table, int num_terms,
                            const double *vA, int64_t vA_len)
{
  try
  {
    if (plan == nullptr)
      return ASGK_ERR_INVALID;
    *plan = nullptr;
    if (n != 3)
      return ASGK_ERR_UNSUPPORTED;
    if (num_terms < 1 || vA == nullptr || table == nullptr || num_cells < 1)
      return ASGK_ERR_INVALID;
    direction_pairs dp;
    if (int rc = build_direction_pairs(d, level, num_cells, table, dp))
      return rc;
    if (vA_len != int64_t(dp.nconn) * d * num_terms * 9)
      return ASGK_ERR_INVALID;
    std::vector<double> B;
    int n_identity = 0;
    std::vector<std::vector<int>> multi;
    if (int rc = global_blocks(d, num_terms, dp.conn_row, dp.conn_col, vA, B,
                               n_identity, multi))
      return rc;
    // entries of dimensions some term acts in
    std::vector<char> used(d, 0);
    for (int64_t j = 0; j < dp.nconn; j++)
      for (int k = 0; k < d; k++)
        for (int e = 0; e < 9; e++)
          if (B[(j * d + k) * 10 + e] != 0.0)
            used[k] = 1;
    std::vector<int64_t> gptr(num_cells + 1, 0);
    std::vector<int> gcol, gkb;
    for (int r = 0; r < num_cells; r++)
    {
      for (int64_t e = dp.ptr[r]; e < dp.ptr[r + 1]; e++)
        if (used[dp.dim[e]])
        {
          gcol.push_back(dp.col[e]);
          gkb.push_back(dp.conn[e] * d + dp.dim[e]);
        }
      gptr[r + 1] = int64_t(gcol.size());
    }
    // the diagonal pairs (one per cell) for the Jacobi preconditioners
    std::vector<int64_t> rp(num_cells + 1);
    std::vector<int> col(num_cells), conn(size_t(num_cells) * d);
    for (int r = 0; r <= num_cells; r++)
      rp[r] = r;
    for (int r = 0; r < num_cells; r++)
    {
      col[r] = r;
      for (int k = 0; k < d; k++)
        conn[size_t(r) * d + k] = dp.self_conn[size_t(r) * d + k];
    }
    if (int rc = build_plan(plan, d, n, num_cells, num_cells, num_terms, rp,
                            col.data(), conn.data(), index_mode::conn, vA, vA_len))
      return rc;
    auto &p = (*plan)->p;
    p.global     = true;
    p.gnnz       = int64_t(gcol.size());
    p.g_identity = n_identity;
    p.g_conn_row = dp.conn_row;
    p.g_conn_col = dp.conn_col;
    int64_t &bytes = p.device_bytes;
    int rc = ASGK_OK;
    if ((rc = dev_alloc(&p.gptr, num_cells + 1, bytes)) ||
        (rc = dev_alloc(&p.gcol, std::max<int64_t>(p.gnnz, 1), bytes)) ||
        (rc = dev_alloc(&p.gkb, std::max<int64_t>(p.gnnz, 1), bytes)) ||
        (rc = dev_alloc(&p.gB64, int64_t(B.size()), bytes)) ||
        (rc = dev_alloc(&p.gB32, int64_t(B.size() / 10 * 12), bytes)))
    {
      asgk_plan_destroy(*plan);
      *plan = nullptr;
      return rc;
    }
    auto up = [&](void *dst, const void *src, size_t b) -> int {
      if (b == 0)
        return ASGK_OK;
      ASGK_CUDA(cudaMemcpy(dst, src, b, cudaMemcpyHostToDevice));
      return ASGK_OK;
    };
    // cells with the most single-direction neighbours first (coarse cells
    // reach every cell of a dimension: up to 2^level per dimension), each
    // cell's list cut into slices of at most global_slice(d) entries
    std::vector<int> order(num_cells);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return (gptr[a + 1] - gptr[a]) > (gptr[b + 1] - gptr[b]);
    });
    std::vector<int> srow, slen, rs0(num_cells), rns(num_cells);
    std::vector<int64_t> sbeg;
    for (int r : order)
    {
      int64_t const e = gptr[r + 1] - gptr[r];
      int const sz    = global_slice(d);
      int const ns    = int(std::max<int64_t>(1, (e + sz - 1) / sz));
      rs0[r] = int(srow.size());
      rns[r] = ns;
      for (int q = 0; q < ns; q++)
      {
        srow.push_back(r);
        sbeg.push_back(gptr[r] + int64_t(q) * sz);
        slen.push_back(int(std::min<int64_t>(sz, e - int64_t(q) * sz)));
      }
    }
    p.gslices = int(srow.size());
    if ((rc = dev_alloc(&p.slice_row, p.gslices, bytes)) ||
        (rc = dev_alloc(&p.slice_len, p.gslices, bytes)) ||
        (rc = dev_alloc(&p.slice_beg, p.gslices, bytes)) ||
        (rc = dev_alloc(&p.row_slice0, num_cells, bytes)) ||
        (rc = dev_alloc(&p.row_nslice, num_cells, bytes)) ||
        (rc = dev_alloc(&p.gscratch, int64_t(p.gslices) * p.tensor, bytes)) ||
        (rc = dev_alloc(&p.gtickets, num_cells, bytes)))
    {
      asgk_plan_destroy(*plan);
      *plan = nullptr;
      return rc;
    }
    // chains of the terms acting in several dimensions
    p.g_multi = multi;
    if (!multi.empty())
    {
      std::vector<std::vector<std::pair<int, int>>> chains;
      std::vector<int> chain_term;
      for (auto const &m : multi)
        for (auto &c : term_chains(std::vector<int>(m.begin() + 1, m.end())))
        {
          chains.push_back(c);
          chain_term.push_back(m[0]);
        }
      p.gchains = int(chains.size());
      int stages = 0;
      for (auto const &c : chains)
        stages = std::max(stages, int(c.size()));
      // per-dimension neighbour lists (every entry of the direction pairs)
      std::vector<int64_t> dptr(size_t(d) * (num_cells + 1), 0);
      std::vector<int> dcol, dconn;
      std::vector<unsigned char> drel;
      std::vector<int64_t> per_dim(d, 0);
      for (int k = 0; k < d; k++)
      {
        for (int r = 0; r < num_cells; r++)
        {
          for (int64_t e = dp.ptr[r]; e < dp.ptr[r + 1]; e++)
            if (dp.dim[e] == k)
            {
              int const j = dp.conn[e];
              dcol.push_back(dp.col[e]);
              dconn.push_back(j);
              drel.push_back(dp.conn_col[j] < dp.conn_row[j] ? 0 : (dp.conn_col[j] == dp.conn_row[j] ? 1 : 2));
            }
          dptr[size_t(k) * (num_cells + 1) + r + 1] = int64_t(dcol.size());
        }
        per_dim[k] = int64_t(dcol.size()) - dptr[size_t(k) * (num_cells + 1)];
        if (k + 1 < d)
          dptr[size_t(k + 1) * (num_cells + 1)] = int64_t(dcol.size());
      }
      std::vector<int4> jobs;
      for (int s = 0; s < stages; s++)
      {
        p.stage_job0.push_back(int(jobs.size()));
        for (int c = 0; c < p.gchains; c++)
          if (int(chains[c].size()) > s)
          {
            jobs.push_back(make_int4(c, chains[c][s].first, chains[c][s].second, chain_term[c]));
            p.gchain_entries += per_dim[chains[c][s].first];
          }
        p.stage_njobs.push_back(int(jobs.size()) - p.stage_job0.back());
      }
      std::vector<int> last(p.gchains);
      for (int c = 0; c < p.gchains; c++)
        last[c] = (int(chains[c].size()) - 1) % 2;
      int64_t const N = int64_t(num_cells) * p.tensor;
      if ((rc = dev_alloc(&p.gjobs, int64_t(jobs.size()), bytes)) ||
          (rc = dev_alloc(&p.gchain_last, p.gchains, bytes)) ||
          (rc = dev_alloc(&p.gd_ptr, int64_t(dptr.size()), bytes)) ||
          (rc = dev_alloc(&p.gd_col, std::max<int64_t>(int64_t(dcol.size()), 1), bytes)) ||
          (rc = dev_alloc(&p.gd_conn, std::max<int64_t>(int64_t(dconn.size()), 1), bytes)) ||
          (rc = dev_alloc(&p.gd_rel, std::max<int64_t>(int64_t(drel.size()), 1), bytes)) ||
          (rc = dev_alloc(&p.gwork, 2 * int64_t(p.gchains) * N, bytes)) ||
          (rc = up(p.gjobs, jobs.data(), sizeof(int4) * jobs.size())) ||
          (rc = up(p.gchain_last, last.data(), sizeof(int) * last.size())) ||
          (rc = up(p.gd_ptr, dptr.data(), sizeof(int64_t) * dptr.size())) ||
          (rc = up(p.gd_col, dcol.data(), sizeof(int) * dcol.size())) ||
          (rc = up(p.gd_conn, dconn.data(), sizeof(int) * dconn.size())) ||
          (rc = up(p.gd_rel, drel.data(), drel.size())))
      {
        asgk_plan_destroy(*plan);
        *plan = nullptr;
        return rc;
      }
    }
    // d >= 5: per-cell dimension segments (the entries of a cell come in
    // dimension order) and two cell orders
    if (d >= 5)
    {
      std::vector<int> seg(size_t(num_cells) * (d + 1));
      std::vector<int> longest(num_cells, 0), total(num_cells, 0);
      for (int r = 0; r < num_cells; r++)
      {
        int64_t e = gptr[r];
        for (int k = 0; k <= d; k++)
        {
          while (e < gptr[r + 1] && gkb[e] % d < k)
            ++e;
          seg[size_t(r) * (d + 1) + k] = int(e - gptr[r]);
        }
        for (int k = 0; k < d; k++)
          longest[r] = std::max(longest[r], seg[size_t(r) * (d + 1) + k + 1] -
                                                seg[size_t(r) * (d + 1) + k]);
        total[r] = seg[size_t(r) * (d + 1) + d];
      }
      // the FP32 kernel's warps take one dimension each (longest segment
      // first), the FP64 kernel's equal ranges (most entries first)
      std::vector<int> corder(2 * size_t(num_cells));
      std::iota(corder.begin(), corder.begin() + num_cells, 0);
      std::iota(corder.begin() + num_cells, corder.end(), 0);
      std::stable_sort(corder.begin(), corder.begin() + num_cells,
                       [&](int a, int b) { return longest[a] > longest[b]; });
      std::stable_sort(corder.begin() + num_cells, corder.end(),
                       [&](int a, int b) { return total[a] > total[b]; });
      if ((rc = dev_alloc(&p.gseg, int64_t(seg.size()), bytes)) ||
          (rc = dev_alloc(&p.gcell_order, 2 * int64_t(num_cells), bytes)) ||
          (rc = dev_alloc(&p.gx32, int64_t(num_cells) * p.tensor, bytes)) ||
          (rc = up(p.gseg, seg.data(), sizeof(int) * seg.size())) ||
          (rc = up(p.gcell_order, corder.data(), sizeof(int) * corder.size())))
      {
        asgk_plan_destroy(*plan);
        *plan = nullptr;
        return rc;
      }
    }
    std::vector<unsigned> zeros(num_cells, 0u);
    if ((rc = up(p.row_order, order.data(), sizeof(int) * order.size())) ||
        (rc = up(p.slice_row, srow.data(), sizeof(int) * srow.size())) ||
        (rc = up(p.slice_len, slen.data(), sizeof(int) * slen.size())) ||
        (rc = up(p.slice_beg, sbeg.data(), sizeof(int64_t) * sbeg.size())) ||
        (rc = up(p.row_slice0, rs0.data(), sizeof(int) * rs0.size())) ||
        (rc = up(p.row_nslice, rns.data(), sizeof(int) * rns.size())) ||
        (rc = up(p.gtickets, zeros.data(), sizeof(unsigned) * zeros.size())) ||
        (rc = up(p.gptr, gptr.data(), sizeof(int64_t) * gptr.size())) ||
        (rc = up(p.gcol, gcol.data(), sizeof(int) * gcol.size())) ||
        (rc = up(p.gkb, gkb.data(), sizeof(int) * gkb.size())) ||
        (rc = upload_global_blocks(p, B)))
    {
      asgk_plan_destroy(*plan);
      *plan = nullptr;
      return rc;
    }
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_plan_info(const asgk_plan *plan, int64_t *num_batch,
                   int64_t *input_size, int64_t *output_size, int64_t *flops,
                   int64_t *device_bytes)
{
  try
  {
    if (!plan)
      return ASGK_ERR_INVALID;
    auto const &p = plan->p;
    if (num_batch)
      *num_batch = p.global ? p.gnnz + p.gchain_entries : p.nnz;
    if (input_size)
      *input_size = int64_t(p.cols) * p.tensor;
    if (output_size)
      *output_size = int64_t(p.rows) * p.tensor;
    // global mode: one contraction in one dimension per entry
    if (flops)
      *flops = p.global ? int64_t(p.tensor) * p.n * (p.gnnz + p.gchain_entries) * 2
                        : int64_t(p.tensor) * p.n * p.d * p.terms * p.nnz * 2;
    if (device_bytes)
      *device_bytes = p.device_bytes + tc_bytes(p.tc);
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_apply(asgk_plan *plan, int precision, double alpha, const double *x,
               double beta, double *y, asgk_stream stream)
{
  try
  {
    if (!plan || !x || !y)
      return ASGK_ERR_INVALID;
    auto &p = plan->p;
    cudaStream_t s = as_stream(stream);
    if (p.terms == 0 || p.nnz == 0 || alpha == 0.0)
    {
      // only the scaling of y remains (src/asgard_kronmult_matrix.hpp:344-349)
      int64_t const ny = int64_t(p.rows) * p.tensor;
      if (beta == 0.0)
        return launch_fill(y, ny, 0.0, s);
      if (beta != 1.0)
        return launch_scale(y, ny, beta, s);
      return ASGK_OK;
    }
    return launch_apply(p, precision, alpha, x, 0, beta, y, 0, 0.0, s);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_apply_f32(asgk_plan *plan, float alpha, const float *x, float beta,
                   float *y, asgk_stream stream)
{
  try
  {
    if (!plan || !x || !y)
      return ASGK_ERR_INVALID;
    auto &p = plan->p;
    if (p.terms == 0 || p.nnz == 0)
      return ASGK_ERR_UNSUPPORTED;
    return launch_apply(p, ASGK_FP32, alpha, x, 1, beta, y, 1, 0.0,
                        as_stream(stream));
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_apply_host(asgk_plan *plan, double alpha, const double *x,
                    double beta, double *y, asgk_stream stream)
{
  try
  {
    if (!plan || !x || !y)
      return ASGK_ERR_INVALID;
    auto &p          = plan->p;
    cudaStream_t s   = as_stream(stream);
    int64_t const nx = int64_t(p.cols) * p.tensor;
    int64_t const ny = int64_t(p.rows) * p.tensor;
    if (p.xw == nullptr)
    {
      int rc = ASGK_OK;
      if ((rc = dev_alloc(&p.xw, std::max<int64_t>(nx, 1), p.device_bytes)) ||
          (rc = dev_alloc(&p.yw, std::max<int64_t>(ny, 1), p.device_bytes)))
      {
        cudaFree(p.xw);
        p.xw = nullptr;
        return rc;
      }
      p.ws_owned = true;
    }
    ASGK_CUDA(cudaMemcpyAsync(p.xw, x, sizeof(double) * nx,
                              cudaMemcpyHostToDevice, s));
    if (beta != 0.0)
      ASGK_CUDA(cudaMemcpyAsync(p.yw, y, sizeof(double) * ny,
                                cudaMemcpyHostToDevice, s));
    if (int rc = asgk_apply(plan, ASGK_FP64, alpha, p.xw, beta, p.yw, stream))
      return rc;
    ASGK_CUDA(cudaMemcpyAsync(y, p.yw, sizeof(double) * ny,
                              cudaMemcpyDeviceToHost, s));
    ASGK_CUDA(cudaStreamSynchronize(s));
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_apply_euler(asgk_plan *plan, int precision, double dt, double alpha,
                     const double *x, double beta, double *y,
                     asgk_stream stream)
{
  try
  {
    if (!plan || !x || !y)
      return ASGK_ERR_INVALID;
    auto &p = plan->p;
    if (p.rows != p.cols)
      return ASGK_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    if (p.terms == 0 || p.nnz == 0 || dt == 0.0)
    {
      int64_t const ny = int64_t(p.rows) * p.tensor;
      if (beta == 0.0)
      {
        if (int rc = launch_copy(y, x, ny, s))
          return rc;
        return launch_scale(y, ny, alpha, s);
      }
      if (int rc = launch_scale(y, ny, beta, s))
        return rc;
      return launch_axpy(y, x, ny, alpha, s);
    }
    return launch_apply(p, precision, -dt * alpha, x, 0, beta, y, 0, alpha, s);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_gmres_dense(int n, const double *A, double *x, const double *b,
                     int restart, int max_outer, double tol,
                     asgk_gmres_info *info)
{
  return asgk_gmres_dense_precond(n, A, x, b, nullptr, restart, max_outer, tol,
                                  info);
}

int asgk_gmres_dense_precond(int n, const double *A, double *x, const double *b,
                             const double *M, int restart, int max_outer,
                             double tol, asgk_gmres_info *info)
{
  try
  {
    if (n <= 0 || !A || !x || !b)
      return ASGK_ERR_INVALID;
    if (restart <= 0)
      restart = asgk_default_gmres_restarts(n);
    if (restart > n)
      return ASGK_ERR_INVALID;
    if (max_outer <= 0)
      max_outer = n;
    if (!(tol > 0))
      tol = 1e-12;
    // the reference's dense_preconditioner (src/solver.cpp:11-38) factors M
    // (getrf) and solves with the factors (getrs) on the left of every
    // residual b - A x and every new basis vector A v -- for device vectors
    // on a host copy (:27-33); the same here: LU with partial pivoting on the
    // host, the product on the device, the solve on the host
    std::vector<double> lu;
    std::vector<int> piv;
    if (M != nullptr)
    {
      lu.assign(M, M + int64_t(n) * n);
      piv.assign(n, 0);
      for (int c = 0; c < n; c++)
      {
        int p = c;
        for (int r = c + 1; r < n; r++)
          if (std::abs(lu[r + int64_t(c) * n]) > std::abs(lu[p + int64_t(c) * n]))
            p = r;
        if (lu[p + int64_t(c) * n] == 0.0 || !std::isfinite(lu[p + int64_t(c) * n]))
          return ASGK_ERR_BREAKDOWN;
        piv[c] = p;
        if (p != c)
          for (int j = 0; j < n; j++)
            std::swap(lu[c + int64_t(j) * n], lu[p + int64_t(j) * n]);
        for (int r = c + 1; r < n; r++)
          lu[r + int64_t(c) * n] /= lu[c + int64_t(c) * n];
        for (int j = c + 1; j < n; j++)
        {
          double const u = lu[c + int64_t(j) * n];
          if (u != 0.0)
            for (int r = c + 1; r < n; r++)
              lu[r + int64_t(j) * n] -= lu[r + int64_t(c) * n] * u;
        }
      }
    }
    std::vector<double> hv(M != nullptr ? n : 0);
    auto lu_solve = [&](double *v) {
      for (int c = 0; c < n; c++)
        if (piv[c] != c)
          std::swap(v[c], v[piv[c]]);
      for (int c = 0; c < n; c++)
        for (int r = c + 1; r < n; r++)
          v[r] -= lu[r + int64_t(c) * n] * v[c];
      for (int c = n - 1; c >= 0; c--)
      {
        v[c] /= lu[c + int64_t(c) * n];
        for (int r = 0; r < c; r++)
          v[r] -= lu[r + int64_t(c) * n] * v[c];
      }
    };
    double *dA = nullptr, *dx = nullptr, *db = nullptr;
    int64_t bytes = 0;
    int rc;
    if ((rc = dev_alloc(&dA, int64_t(n) * n, bytes)) ||
        (rc = dev_alloc(&dx, n, bytes)) || (rc = dev_alloc(&db, n, bytes)))
    {
      cudaFree(dA);
      cudaFree(dx);
      cudaFree(db);
      return rc;
    }
    cudaStream_t s = nullptr;
    gmres_ws ws;
    core_stats st;
    // y = beta*y + alpha*A*x, then y = M^-1 y with a preconditioner
    auto mat = [&](double a, const double *xin, double bb, double *yout,
                   cudaStream_t ss) -> int {
      k_dense_gemv<<<(n + 3) / 4, 128, 0, ss>>>(n, dA, a, xin, bb, yout);
      ASGK_LAUNCHED();
      if (M == nullptr)
        return ASGK_OK;
      ASGK_CUDA(cudaMemcpyAsync(hv.data(), yout, sizeof(double) * n,
                                cudaMemcpyDeviceToHost, ss));
      ASGK_CUDA(cudaStreamSynchronize(ss));
      lu_solve(hv.data());
      ASGK_CUDA(cudaMemcpyAsync(yout, hv.data(), sizeof(double) * n,
                                cudaMemcpyHostToDevice, ss));
      ASGK_CUDA(cudaStreamSynchronize(ss));
      return ASGK_OK;
    };
    rc = ASGK_OK;
    if (cudaMemcpy(dA, A, sizeof(double) * n * int64_t(n), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(db, b, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
    if (rc == ASGK_OK)
      rc = gmres_core(ws, n, mat, nullptr, dx, db, restart, max_outer, tol, st, s);
    if (rc == ASGK_OK &&
        cudaMemcpy(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
    cudaFree(dA);
    cudaFree(dx);
    cudaFree(db);
    if (rc == ASGK_OK && info)
    {
      *info              = asgk_gmres_info{};
      info->error        = st.err;
      info->iterations   = st.total;
      info->status       = st.status;
      info->outer_steps  = st.restarts;
      info->matvecs_fp64 = st.matvecs;
    }
    return rc;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_cgs_step(const double *V, int64_t ldv, int k, double *w, int64_t n,
                  double *h, double *norm, asgk_stream stream)
{
  try
  {
    if (!V || !w || !h || !norm || k < 1 || n < 1 || ldv < n)
      return ASGK_ERR_INVALID;
    cudaStream_t s   = as_stream(stream);
    int const blocks = max_reduction_blocks();
    double *part     = nullptr;
    size_t const cnt = size_t(blocks) * (k + 1) + 1;
    ASGK_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&part),
                              sizeof(double) * cnt, s));
    double *nrm2 = part + size_t(blocks) * (k + 1);
    int used     = 0;
    int rc       = launch_multidot(V, ldv, k, w, n, part, &used, s);
    if (!rc)
      rc = launch_reduce_parts(part, used, k, h, s);
    if (!rc)
      rc = launch_update_norm(V, ldv, k, h, w, n, part, &used, s);
    if (!rc)
      rc = launch_reduce_parts(part, used, 1, nrm2, s);
    double host = 0;
    if (!rc && cudaMemcpyAsync(&host, nrm2, sizeof(double),
                               cudaMemcpyDeviceToHost, s) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
    if (cudaFreeAsync(part, s) != cudaSuccess && !rc)
      rc = ASGK_ERR_CUDA;
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
    if (!rc)
      *norm = std::sqrt(host);
    return rc;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_default_gmres_restarts(int64_t n)
{
  int const minimum = int(std::min<int64_t>(10, n));
  int const maximum = int(std::min<int64_t>(200, n));
  double const MB   = double(n) * sizeof(double) / 1048576.0;
  int const want    = int(512.0 / MB);
  return std::clamp(want, minimum, maximum);
}

} // extern "C"

namespace asgk
{
// The solve behind asgk_gmres_euler*: pc (or nullptr) is the right
// preconditioner of the flexible GMRES, given whether the inner operator is
// the low-precision one.
using make_pc_t = std::function<precond_t(bool low)>;

// pc_serial identifies the preconditioner for the recorded-cycle cache (0:
// none); pc_graph_ok says whether its launches may be recorded.
int gmres_euler_impl(asgk_plan *plan, double dt, double *x, const double *b,
                     int restart, int max_outer, double tol, int tol_mode,
                     int precision, make_pc_t const *make_pc,
                     asgk_gmres_info *info, asgk_stream stream,
                     uint64_t pc_serial = 0, bool pc_graph_ok = false)
{
  if (!plan || !x || !b)
    return ASGK_ERR_INVALID;
  auto &p = plan->p;
  if (p.rows != p.cols)
    return ASGK_ERR_INVALID;
  if (precision != ASGK_FP64 && precision != ASGK_FP32 && precision != ASGK_BF16)
    return ASGK_ERR_UNSUPPORTED;
  // the tensor-core operator exists for global plans; its set-up (host work,
  // allocations) happens here, before any cycle is recorded
  if (precision == ASGK_BF16)
    if (int rc = tc_prepare(p))
      return rc;
  int64_t const n = int64_t(p.rows) * p.tensor;
  if (restart <= 0)
    restart = asgk_default_gmres_restarts(n);
  if (restart > n)
    return ASGK_ERR_INVALID; // src/solver.cpp:175-181
  if (max_outer <= 0)
    max_outer = int(std::min<int64_t>(n, 1 << 30));
  if (!(tol > 0))
    tol = 1e-12; // src/solver.cpp:165-166 default for double
  cudaStream_t s = as_stream(stream);
  auto *ex       = extras_of(plan, true);
  gmres_ws &ws   = ex->ws;

  asgk_gmres_info out{};
  auto op64 = [&](double a, const double *xin, double bb, double *yout,
                  cudaStream_t ss) -> int {
    return asgk_apply_euler(plan, ASGK_FP64, dt, a, xin, bb, yout, ss);
  };
  auto oplow = [&](double a, const double *xin, double bb, double *yout,
                   cudaStream_t ss) -> int {
    return asgk_apply_euler(plan, precision, dt, a, xin, bb, yout, ss);
  };
  precond_t pcf;
  precond_t const *pcp = nullptr;
  if (make_pc != nullptr)
  {
    pcf = (*make_pc)(precision != ASGK_FP64);
    pcp = &pcf;
  }
  bool const precond = pcp != nullptr;

  double bnorm = 0;
  if (ws.ensure(n, restart, pcp != nullptr) != ASGK_OK)
    return ASGK_ERR_ALLOC;
  if (int rc = norm2(ws, b, n, bnorm, s))
    return rc;
  double const tol_abs = (tol_mode == ASGK_TOL_REL) ? tol * bnorm : tol;

  // recorded cycles take several Arnoldi steps per graph node when every
  // kernel of a step reads the gate: the global operator without chains
  // (one kernel), a Jacobi preconditioner or none, the Krylov kernels
  int const node_steps =
      (p.global && p.gchains == 0 && p.terms > 0 && p.nnz > 0 && dt != 0.0)
          ? g_gmres_node_steps
          : 1;

  core_stats st;
  int status = ASGK_OK;
  double true_res = -1; // FP64 residual of the final x when already known
  if (precision == ASGK_FP64 && !precond)
  {
    graph_key const gk{plan, dt, ASGK_FP64, 0, restart, false, node_steps};
    if (int rc = gmres_core(ws, n, op64, nullptr, x, b, restart, max_outer,
                            tol_abs, st, s, tol_mode == ASGK_TOL_REL, &gk))
      return rc;
    out.error        = st.err;
    out.iterations   = st.total;
    out.outer_steps  = st.restarts;
    out.matvecs_fp64 = st.matvecs;
    status           = st.status;
    if (st.verified)
      true_res = st.err;
  }
  else
  {
    // FP64 iterative refinement: r = b - A x in FP64, inner (flexible) GMRES
    // on A e = r with the low-precision operator, x += e.
    // inner tolerances: about the operator's rounding (FP32 2^-24, BF16
    // operands 2^-9), below which an inner solve gains nothing
    double const inner_rtol =
        (precision == ASGK_FP64) ? 1e-10 : (precision == ASGK_FP32 ? 1e-5 : g_bf16_inner_rtol);
    int total = 0, low = 0, fp64 = 0, pcalls = 0, steps = 0, fallback = 0;
    double rnorm = 0, prev_rnorm = 0;
    int const max_steps = 50;
    precond_t const *use_pc = pcp;
    status = ASGK_ERR_NOT_CONVERGED;
    for (;;)
    {
      // a zero initial guess (||x|| = 0) needs no product: r = b
      bool x_zero = false;
      if (steps == 0)
      {
        double xn = 0;
        if (int rc = norm2(ws, x, n, xn, s))
          return rc;
        x_zero = (xn == 0.0);
      }
      if (int rc = launch_copy(ws.r, b, n, s))
        return rc;
      if (!x_zero)
      {
        if (int rc = op64(-1.0, x, 1.0, ws.r, s))
          return rc;
        ++fp64;
      }
      if (int rc = norm2(ws, ws.r, n, rnorm, s))
        return rc;
      if (!std::isfinite(rnorm))
      {
        status = ASGK_ERR_NONFINITE;
        break;
      }
      if (rnorm <= tol_abs)
      {
        status   = ASGK_OK;
        true_res = rnorm;
        break;
      }
      if (steps >= max_steps || total >= max_outer * (restart + 1))
        break;
      // The learned preconditioner is dropped (plain GMRES from the current
      // iterate) when a refinement step did not halve the FP64 residual.
      if (use_pc && steps > 0 && rnorm > 0.5 * prev_rnorm)
      {
        use_pc   = nullptr;
        fallback = 1;
      }
      prev_rnorm = rnorm;
      if (int rc = launch_fill(ws.e, n, 0.0, s))
        return rc;
      core_stats ist;
      double const itol = std::max(inner_rtol * rnorm, 0.5 * tol_abs);
      int const inner_outer = std::max(1, max_outer);
      // FP32 inner solves: Gram-Schmidt over an FP32 copy of the basis
      bool const low_basis = (precision != ASGK_FP64) && g_gmres_low_basis;
      graph_key const gk{plan, dt, precision, use_pc ? pc_serial : 0, restart,
                         low_basis, node_steps, use_pc != nullptr && g_gmres_fused_copy};
      bool const recordable = (use_pc == nullptr || pc_graph_ok);
      if (int rc = gmres_core(ws, n, (precision == ASGK_FP64) ? matvec_t(op64) : matvec_t(oplow),
                              use_pc, ws.e, ws.r, restart, inner_outer, itol, ist, s,
                              false, recordable ? &gk : nullptr, low_basis))
        return rc;
      total += ist.total;
      if (precision == ASGK_FP64)
        fp64 += ist.matvecs;
      else
        low += ist.matvecs;
      pcalls += ist.pcalls;
      ++steps;
      if (ist.stagnated && use_pc)
      {
        // keep the progress made (e is a valid correction), then continue
        // without the learned preconditioner
        if (int rc = launch_axpy(x, ws.e, n, 1.0, s))
          return rc;
        use_pc   = nullptr;
        fallback = 1;
        continue;
      }
      if (ist.status == ASGK_ERR_NONFINITE)
      {
        if (use_pc)
        {
          // a non-finite network output: retry the step without it
          use_pc   = nullptr;
          fallback = 1;
          continue;
        }
        status = ASGK_ERR_NONFINITE;
        break;
      }
      if (int rc = launch_axpy(x, ws.e, n, 1.0, s))
        return rc;
    }
    out.error        = rnorm;
    out.iterations   = total;
    out.outer_steps  = steps;
    out.matvecs_low  = low;
    out.matvecs_fp64 = fp64;
    out.precond_calls = pcalls;
    out.fallback      = fallback;
  }
  // FP64 check of the final iterate (unless the solve ended on one)
  double rfinal = true_res;
  if (rfinal < 0)
  {
    if (int rc = launch_copy(ws.r, b, n, s))
      return rc;
    if (int rc = op64(-1.0, x, 1.0, ws.r, s))
      return rc;
    if (int rc = norm2(ws, ws.r, n, rfinal, s))
      return rc;
  }
  out.true_relres = (bnorm > 0) ? rfinal / bnorm : rfinal;
  out.status      = status;
  if (info)
    *info = out;
  return ASGK_OK;
}

} // namespace asgk

extern "C"
{

int asgk_gmres_euler(asgk_plan *plan, double dt, double *x, const double *b,
                     int restart, int max_outer, double tol, int tol_mode,
                     int precision, asgk_mlp *precond, asgk_gmres_info *info,
                     asgk_stream stream)
{
  try
  {
    if (precond == nullptr)
      return gmres_euler_impl(plan, dt, x, b, restart, max_outer, tol, tol_mode,
                              precision, nullptr, info, stream);
    cudaStream_t s = as_stream(stream);
    make_pc_t const mk = [&](bool low) -> precond_t {
      return [=](double *v, double *z, const double *sc, float *vc,
                 cudaStream_t ss) -> int {
        int64_t const nn = int64_t(plan->p.rows) * plan->p.tensor;
        if (vc)
        {
          if (int rc = launch_store_basis(v, vc, nn, sc, 1.0, ss))
            return rc;
        }
        else if (sc)
          if (int rc = launch_scale_by(v, nn, sc, ss))
            return rc;
        return mlp_precondition(precond, plan, v, z, ss, low);
      };
    };
    return gmres_euler_impl(plan, dt, x, b, restart, max_outer, tol, tol_mode,
                            precision, &mk, info, stream);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_gmres_euler_jacobi(asgk_plan *plan, double dt, double *x,
                            const double *b, int restart, int max_outer,
                            double tol, int tol_mode, int precision,
                            asgk_jacobi *precond, asgk_gmres_info *info,
                            asgk_stream stream)
{
  try
  {
    if (precond == nullptr || plan == nullptr)
      return ASGK_ERR_INVALID;
    // a preconditioner of another shape would index past v and z
    if (int rc = jacobi_check_shape(precond, plan->p.rows, plan->p.tensor))
      return rc;
    cudaStream_t s = as_stream(stream);
    // with the FP32 global apply at d >= 5 next, the line preconditioner
    // also writes the FP32 copy of its output that apply reads
    plan_data const &pp = plan->p;
    float *zc = (precision == ASGK_FP32 && pp.gx32 != nullptr && g_gmres_fused_copy &&
                 jacobi_writes_zcopy(precond))
                    ? pp.gx32
                    : nullptr;
    make_pc_t const mk = [&](bool low) -> precond_t {
      return [=, &pp](double *v, double *z, const double *sc, float *vc,
                      cudaStream_t ss) -> int {
        float *c = low ? zc : nullptr;
        int const rc = jacobi_apply_handle(precond, low, v, z, sc, vc, ss, c);
        if (rc == ASGK_OK && c != nullptr)
          pp.gx32_src = z;
        return rc;
      };
    };
    return gmres_euler_impl(plan, dt, x, b, restart, max_outer, tol, tol_mode,
                            precision, &mk, info, stream, jacobi_serial(precond),
                            true);
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_gmres_euler_f32(asgk_plan *plan, float dt, float *x, const float *b,
                         int restart, int max_outer, float tol,
                         asgk_gmres_info *info, asgk_stream stream)
{
  try
  {
    if (!plan || !x || !b)
      return ASGK_ERR_INVALID;
    int64_t const n = int64_t(plan->p.rows) * plan->p.tensor;
    if (plan->p.rows != plan->p.cols)
      return ASGK_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    double *w      = nullptr;
    int64_t unused = 0;
    if (int rc = dev_alloc(&w, std::max<int64_t>(2 * n, 1), unused))
      return rc;
    double *xd = w, *bd = w + n;
    int const blocks = int(std::min<int64_t>((n + 255) / 256, 65535));
    k_widen<<<blocks, 256, 0, s>>>(n, x, xd);
    k_widen<<<blocks, 256, 0, s>>>(n, b, bd);
    int rc = cudaGetLastError() == cudaSuccess ? ASGK_OK : ASGK_ERR_CUDA;
    count_launch(2);
    if (rc == ASGK_OK)
      rc = gmres_euler_impl(plan, double(dt), xd, bd, restart, max_outer,
                            tol > 0 ? double(tol) : 1e-6, ASGK_TOL_ABS,
                            ASGK_FP32, nullptr, info, stream);
    if (rc == ASGK_OK)
    {
      k_narrow<<<blocks, 256, 0, s>>>(n, xd, x);
      rc = cudaGetLastError() == cudaSuccess ? ASGK_OK : ASGK_ERR_CUDA;
      count_launch(1);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess && rc == ASGK_OK)
      rc = ASGK_ERR_CUDA;
    cudaFree(w);
    return rc;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_set_gmres_graphs(int enable)
{
  int const old  = g_gmres_graphs ? 1 : 0;
  g_gmres_graphs = (enable != 0);
  return old;
}

int asgk_set_gmres_node_steps(int steps)
{
  int const old = g_gmres_node_steps;
  if (steps >= 1)
    g_gmres_node_steps = steps;
  return old;
}

int asgk_set_gmres_basis(int fp32)
{
  int const old     = g_gmres_low_basis ? 1 : 0;
  g_gmres_low_basis = (fp32 != 0);
  return old;
}

int asgk_set_gmres_fused_copy(int on)
{
  int const old      = g_gmres_fused_copy ? 1 : 0;
  g_gmres_fused_copy = (on != 0);
  return old;
}

double asgk_set_bf16_inner_tol(double rtol)
{
  double const old = g_bf16_inner_rtol;
  if (rtol > 0 && rtol < 1)
    g_bf16_inner_rtol = rtol;
  return old;
}

int asgk_implicit_advance(asgk_plan *plan, double dt, double *x, int steps,
                          const double *forcing, int64_t forcing_stride,
                          int restart, int max_outer, double tol, int tol_mode,
                          int precision, int pc_kind, void *precond,
                          asgk_gmres_info *info, asgk_stream stream)
{
  try
  {
    if (!plan || !x || steps < 0 || (steps > 0 && !info) || forcing_stride < 0 ||
        pc_kind < 0 || pc_kind > 2 || (pc_kind != 0 && !precond))
      return ASGK_ERR_INVALID;
    auto &p = plan->p;
    if (p.rows != p.cols)
      return ASGK_ERR_INVALID;
    int64_t const n = int64_t(p.rows) * p.tensor;
    if (forcing && forcing_stride != 0 && forcing_stride < n)
      return ASGK_ERR_INVALID;
    // a preconditioner of another shape is refused before any launch
    if ((pc_kind == 1 &&
         jacobi_check_shape(static_cast<asgk_jacobi *>(precond), p.rows, p.tensor)) ||
        (pc_kind == 2 &&
         mlp_check_shape(static_cast<asgk_mlp *>(precond), p.rows, p.tensor)))
      return ASGK_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    double *b      = nullptr;
    int64_t unused = 0;
    if (int rc = dev_alloc(&b, std::max<int64_t>(n, 1), unused))
      return rc;
    int status = ASGK_OK;
    for (int k = 0; k < steps && status == ASGK_OK; k++)
    {
      // right-hand side x + dt * f(t + dt); the solve starts from it, as the
      // reference starts from a copy of its right-hand side
      if (forcing)
        status = launch_axpy(x, forcing + k * forcing_stride, n, dt, s);
      if (status == ASGK_OK)
        status = launch_copy(b, x, n, s);
      if (status != ASGK_OK)
        break;
      if (pc_kind == 1)
        status = asgk_gmres_euler_jacobi(plan, dt, x, b, restart, max_outer, tol,
                                         tol_mode, precision,
                                         static_cast<asgk_jacobi *>(precond),
                                         info + k, stream);
      else
        status = asgk_gmres_euler(plan, dt, x, b, restart, max_outer, tol,
                                  tol_mode, precision,
                                  static_cast<asgk_mlp *>(pc_kind == 2 ? precond : nullptr),
                                  info + k, stream);
    }
    cudaStreamSynchronize(s);
    cudaFree(b);
    return status;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_imex_advance(asgk_plan *explicit_plan, asgk_plan *implicit_plan,
                      double dt, double *x, int steps, int restart,
                      int max_outer, double tol, int tol_mode, int precision,
                      asgk_jacobi *pc_stage1, asgk_jacobi *pc_stage2,
                      asgk_imex_hook hook, void *hook_ctx, double *work,
                      asgk_gmres_info *info, asgk_stream stream)
{
  try
  {
    if (!explicit_plan || !x || steps < 0 || (steps > 0 && !info))
      return ASGK_ERR_INVALID;
    auto const &pe = explicit_plan->p;
    if (pe.rows != pe.cols)
      return ASGK_ERR_INVALID;
    int64_t const n = int64_t(pe.rows) * pe.tensor;
    if (implicit_plan &&
        int64_t(implicit_plan->p.rows) * implicit_plan->p.tensor != n)
      return ASGK_ERR_INVALID;
    // each stage's preconditioner must fit the implicit plan and invert
    // I - dt*K for that stage's step: dt (stage 1) and dt/2 (stage 2)
    for (int st = 0; st < 2; st++)
    {
      asgk_jacobi *pc = st == 0 ? pc_stage1 : pc_stage2;
      if (pc == nullptr)
        continue;
      if (!implicit_plan ||
          jacobi_check_shape(pc, implicit_plan->p.rows, implicit_plan->p.tensor) ||
          jacobi_dt(pc) != (st == 0 ? dt : 0.5 * dt))
        return ASGK_ERR_INVALID;
    }
    cudaStream_t s = as_stream(stream);
    // f_0, the explicit product, f_1 (then f_1 + dt E f_1), the stage-1
    // solution (then the stage-2 solve's iterate)
    double *owned = nullptr;
    int64_t unused = 0;
    int status     = ASGK_OK;
    if (!work)
    {
      if ((status = dev_alloc(&owned, std::max<int64_t>(4 * n, 1), unused)))
        return status;
      work = owned;
    }
    double *const f0 = work, *const fx = work + n, *const f1 = work + 2 * n,
                  *const f1s = work + 3 * n;
    auto call_hook = [&](int k, int stage, int event, const double *f) -> int {
      return hook ? hook(hook_ctx, k, stage, event, f, stream) : ASGK_OK;
    };
    auto solve = [&](double h, asgk_jacobi *pc, double *xs, const double *b,
                     asgk_gmres_info *out) -> int {
      if (pc)
        return asgk_gmres_euler_jacobi(implicit_plan, h, xs, b, restart, max_outer,
                                       tol, tol_mode, precision, pc, out, stream);
      return asgk_gmres_euler(implicit_plan, h, xs, b, restart, max_outer, tol,
                              tol_mode, precision, nullptr, out, stream);
    };
    for (int k = 0; k < steps && status == ASGK_OK; k++)
    {
      asgk_gmres_info *i1 = info + 2 * k, *i2 = info + 2 * k + 1;
      *i1 = asgk_gmres_info{};
      *i2 = asgk_gmres_info{};
      // stage 1: f_1s = f_0 + dt E f_0 (in x), f_1 from it
      if ((status = launch_copy(f0, x, n, s)) ||
          (status = call_hook(k, 0, ASGK_IMEX_BEFORE_EXPLICIT, x)) ||
          (status = asgk_apply(explicit_plan, ASGK_FP64, 1.0, x, 0.0, fx, stream)) ||
          (status = launch_axpy(x, fx, n, dt, s)) ||
          (status = call_hook(k, 0, ASGK_IMEX_BEFORE_IMPLICIT, x)) ||
          (status = launch_copy(f1, x, n, s)))
        break;
      if (implicit_plan)
      {
        if ((status = solve(dt, pc_stage1, f1, x, i1)) ||
            (status = launch_copy(f1s, f1, n, s)))
          break;
      }
      // stage 2: f_2s = (f_0 + f_1 + dt E f_1) / 2 (in x), f_2 from it
      if ((status = launch_copy(x, f0, n, s)) ||
          (status = call_hook(k, 1, ASGK_IMEX_BEFORE_EXPLICIT, f1)) ||
          (status = asgk_apply(explicit_plan, ASGK_FP64, 1.0, f1, 0.0, fx, stream)) ||
          (status = launch_axpy(f1, fx, n, dt, s)) ||
          (status = launch_axpy(x, f1, n, 1.0, s)) ||
          (status = launch_scale(x, n, 0.5, s)) ||
          (status = call_hook(k, 1, ASGK_IMEX_BEFORE_IMPLICIT, x)))
        break;
      if (implicit_plan)
      {
        if ((status = solve(0.5 * dt, pc_stage2, f1s, x, i2)) ||
            (status = launch_copy(x, f1s, n, s)))
          break;
      }
    }
    cudaStreamSynchronize(s);
    cudaFree(owned);
    return status;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

} // extern "C"
