// Jacobi preconditioners of the backward-Euler operator I - dt*K.
//
// point: the reference's diagonal preconditioner (build_preconditioner,
//   src/asgard_kronmult_matrix.cpp:1015-1067, applied by
//   apply_diagonal_precond, src/solver.cpp:76-91): for every degree of freedom
//   i of cell c, pc_i = sum_t prod_k A_{t,k}(i_k, i_k) over the factors of
//   the cell's own (diagonal) pair, and z_i = v_i / (1 - dt*pc_i).
// block: the inverse of the whole n^d x n^d diagonal block of I - dt*K of
//   each cell, (I - dt * sum_t (x)_k A_{t,k})^{-1} over the diagonal pair's
//   factors, built and inverted on the device (Gauss-Jordan, partial
//   pivoting, one CTA per cell) and applied as a batched block product.  A
//   cell-local map that contains the point preconditioner as its diagonal.
#include "internal.cuh"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <new>

namespace asgk
{
namespace
{
// index of the pair (row, row) in the row's pair list, or -1
__device__ int64_t find_self_pair(const int64_t *row_ptr, const int *col,
                                  int row)
{
  __shared__ long long found;
  if (threadIdx.x == 0)
    found = -1;
  __syncthreads();
  for (int64_t p = row_ptr[row] + threadIdx.x; p < row_ptr[row + 1];
       p += blockDim.x)
    if (col[p] == row)
      atomicMax(&found, (long long)p);
  __syncthreads();
  return found;
}

// offset of the factor A_{t,k} of pair p (column-major n x n block)
__device__ int64_t factor_offset(index_mode mode, const int *idx, int64_t p,
                                 int d, int T, int n, int t, int k)
{
  if (mode == index_mode::conn)
    return int64_t(idx[p * d + k]) * d * T * n * n + int64_t(t * d + k) * n * n;
  return idx[(p * T + t) * d + k];
}

// K_cc(i, j) = sum_t prod_k A_{t,k}(i_k, j_k), dimension 0 slowest
__device__ double diag_block_entry(int i, int j, int d, int n, int T,
                                   index_mode mode, const int *idx,
                                   const double *vA, int64_t p)
{
  double s = 0.0;
  for (int t = 0; t < T; t++)
  {
    double a = 1.0;
    int ii = i, jj = j;
    for (int k = d - 1; k >= 0; k--)
    {
      int const ik = ii % n, jk = jj % n;
      ii /= n;
      jj /= n;
      a *= vA[factor_offset(mode, idx, p, d, T, n, t, k) + ik + jk * n];
    }
    s += a;
  }
  return s;
}

__global__ void k_point_jacobi(int rows, int d, int n, int ts, int T,
                               index_mode mode, const int64_t *row_ptr,
                               const int *col, const int *idx,
                               const double *vA, double dt, double *inv_diag,
                               int *err)
{
  int const row   = blockIdx.x;
  int64_t const p = find_self_pair(row_ptr, col, row);
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
  {
    if (p < 0)
    {
      // no diagonal pair: K_cc = 0
      inv_diag[int64_t(row) * ts + i] = 1.0;
      continue;
    }
    double const den = 1.0 - dt * diag_block_entry(i, i, d, n, T, mode, idx, vA, p);
    if (den == 0.0 || !isfinite(den))
      atomicExch(err, 1);
    inv_diag[int64_t(row) * ts + i] = 1.0 / den;
  }
}

// Gauss-Jordan inverse of I - dt*K_cc in shared memory ([B | I], ts x 2ts,
// row-major), result stored column-major per cell: M[c][j][i] = inv(i, j)
__global__ void k_block_jacobi(int rows, int d, int n, int ts, int T,
                               index_mode mode, const int64_t *row_ptr,
                               const int *col, const int *idx,
                               const double *vA, double dt, double *M,
                               __half *M16, int ps16, int *err)
{
  extern __shared__ double aug[]; // ts x 2ts
  __shared__ int piv;
  int const row   = blockIdx.x;
  int const w     = 2 * ts;
  int64_t const p = find_self_pair(row_ptr, col, row);
  for (int e = threadIdx.x; e < ts * ts; e += blockDim.x)
  {
    int const i = e / ts, j = e - (e / ts) * ts;
    double k = (p >= 0) ? diag_block_entry(i, j, d, n, T, mode, idx, vA, p) : 0.0;
    aug[i * w + j]      = (i == j ? 1.0 : 0.0) - dt * k;
    aug[i * w + ts + j] = (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  bool singular = false;
  for (int c = 0; c < ts; c++)
  {
    if (threadIdx.x == 0)
    {
      int best = c;
      double bv = fabs(aug[c * w + c]);
      for (int r = c + 1; r < ts; r++)
        if (fabs(aug[r * w + c]) > bv)
        {
          bv   = fabs(aug[r * w + c]);
          best = r;
        }
      piv = (bv > 0.0 && isfinite(bv)) ? best : -1;
    }
    __syncthreads();
    if (piv < 0)
    {
      singular = true;
      break;
    }
    if (piv != c)
      for (int j = threadIdx.x; j < w; j += blockDim.x)
      {
        double const t = aug[c * w + j];
        aug[c * w + j]   = aug[piv * w + j];
        aug[piv * w + j] = t;
      }
    __syncthreads();
    double const inv = 1.0 / aug[c * w + c];
    __syncthreads();
    for (int j = threadIdx.x; j < w; j += blockDim.x)
      aug[c * w + j] *= inv;
    __syncthreads();
    for (int e = threadIdx.x; e < ts * w; e += blockDim.x)
    {
      int const r = e / w, j = e - (e / w) * w;
      if (r != c && j != c)
        aug[r * w + j] -= aug[r * w + c] * aug[c * w + j];
    }
    __syncthreads();
    for (int r = threadIdx.x; r < ts; r += blockDim.x)
      if (r != c)
        aug[r * w + c] = 0.0;
    __syncthreads();
  }
  if (singular)
  {
    if (threadIdx.x == 0)
      atomicExch(err, 1);
    return;
  }
  double *Mc = M + int64_t(row) * ts * ts;
  __half *Mh = M16 + int64_t(row) * ps16;
  for (int e = threadIdx.x; e < ps16; e += blockDim.x)
  {
    if (e >= ts * ts)
    {
      Mh[e] = __float2half_rn(0.0f); // padding to a 16-byte multiple
      continue;
    }
    int const j = e / ts, i = e - (e / ts) * ts; // column-major
    double const v = aug[i * w + ts + j];
    Mc[e] = v;
    Mh[e] = __float2half_rn(float(v));
  }
}

__device__ __forceinline__ double to_d(double v) { return v; }
__device__ __forceinline__ double to_d(float v) { return v; }
__device__ __forceinline__ double to_d(__half v) { return __half2float(v); }

// z_c = M_c v_c, one CTA per cell; M column-major so the threads of a CTA
// read consecutive entries
template<typename TM>
__global__ void k_block_apply(int rows, int ts, const TM *__restrict__ M,
                              double *__restrict__ v,
                              double *__restrict__ z,
                              const double *__restrict__ scale_state)
{
  extern __shared__ double vs[];
  int const row = blockIdx.x;
  if (scale_state)
  {
    double const f = scale_state[1];
    for (int i = threadIdx.x; i < ts; i += blockDim.x)
    {
      double const vv          = v[int64_t(row) * ts + i] * f;
      v[int64_t(row) * ts + i] = vv;
      vs[i]                    = vv;
    }
  }
  else
    for (int i = threadIdx.x; i < ts; i += blockDim.x)
      vs[i] = v[int64_t(row) * ts + i];
  __syncthreads();
  const TM *Mc = M + int64_t(row) * ts * ts;
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
  {
    double s = 0.0;
    for (int j = 0; j < ts; j++)
      s = fma(to_d(Mc[int64_t(j) * ts + i]), vs[j], s);
    z[int64_t(row) * ts + i] = s;
  }
}

// FP16 inverses (the FP32 solves' preconditioner): z_c = M_c v_c with the
// cell's block (ps halves, ps a multiple of 8 so every block starts on 16
// bytes) streamed into shared memory by 16-byte loads, all issued before the
// first is used, and FP32 accumulation (the FP16 entries carry ~5e-4
// relative error; the sums add ~1e-7).  Blocks are read once per apply:
// evict-first loads keep L2 for the Krylov basis.
constexpr int kApply16Threads = 128;
constexpr int kApply16Loads   = 8; // 16-byte loads per thread: ps <= 8192

__global__ void __launch_bounds__(kApply16Threads)
    k_block_apply16(int ts, int ps, const __half *__restrict__ M,
                    double *__restrict__ v, double *__restrict__ z,
                    const double *__restrict__ scale_state)
{
  extern __shared__ __align__(16) unsigned char smem16[];
  __half *Ms = reinterpret_cast<__half *>(smem16);
  float *vs  = reinterpret_cast<float *>(smem16 + sizeof(__half) * ps);
  int const row = blockIdx.x;
  int const nv  = ps / 8;
  const uint4 *src = reinterpret_cast<const uint4 *>(M + int64_t(row) * ps);
  uint4 r[kApply16Loads];
#pragma unroll
  for (int l = 0; l < kApply16Loads; l++)
  {
    int const e = threadIdx.x + l * kApply16Threads;
    if (e < nv)
      r[l] = __ldcs(src + e);
  }
  if (scale_state)
  {
    double const f = scale_state[1];
    for (int i = threadIdx.x; i < ts; i += kApply16Threads)
    {
      double const vv          = v[int64_t(row) * ts + i] * f;
      v[int64_t(row) * ts + i] = vv;
      vs[i]                    = static_cast<float>(vv);
    }
  }
  else
    for (int i = threadIdx.x; i < ts; i += kApply16Threads)
      vs[i] = static_cast<float>(v[int64_t(row) * ts + i]);
  uint4 *dst = reinterpret_cast<uint4 *>(Ms);
#pragma unroll
  for (int l = 0; l < kApply16Loads; l++)
  {
    int const e = threadIdx.x + l * kApply16Threads;
    if (e < nv)
      dst[e] = r[l];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < ts; i += kApply16Threads)
  {
    float s0 = 0.0f, s1 = 0.0f;
    int j = 0;
    for (; j + 2 <= ts; j += 2)
    {
      s0 = fmaf(__half2float(Ms[j * ts + i]), vs[j], s0);
      s1 = fmaf(__half2float(Ms[(j + 1) * ts + i]), vs[j + 1], s1);
    }
    if (j < ts)
      s0 = fmaf(__half2float(Ms[j * ts + i]), vs[j], s0);
    z[int64_t(row) * ts + i] = static_cast<double>(s0 + s1);
  }
}

__global__ void k_point_apply(int64_t n, const double *__restrict__ inv_diag,
                              double *__restrict__ v,
                              double *__restrict__ z,
                              const double *__restrict__ scale_state)
{
  double const f = scale_state ? scale_state[1] : 1.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    double vv = v[i];
    if (scale_state)
    {
      vv   = vv * f;
      v[i] = vv;
    }
    z[i] = vv * inv_diag[i];
  }
}

} // namespace

struct jacobi_data
{
  uint64_t serial = 0; // unique per preconditioner built in this process
  int kind  = 0;
  int rows  = 0;
  int ts    = 0;
  double dt = 0;
  double *inv_diag = nullptr; // point: rows*ts
  double *M64      = nullptr; // block: rows*ts*ts, column-major per cell
  __half *M16      = nullptr; // applied inside the FP32 solves, ps16 per cell
  int ps16         = 0;       // ts*ts rounded up to a multiple of 8
  int64_t device_bytes = 0;
  ~jacobi_data()
  {
    cudaFree(inv_diag);
    cudaFree(M64);
    cudaFree(M16);
  }
};

int jacobi_build(plan_data const &p, double dt, int kind, jacobi_data &jd)
{
  if (p.rows != p.cols)
    return ASGK_ERR_INVALID;
  if (kind != ASGK_JACOBI_POINT && kind != ASGK_JACOBI_BLOCK)
    return ASGK_ERR_INVALID;
  int const ts = p.tensor;
  if (kind == ASGK_JACOBI_BLOCK && ts > 81)
    return ASGK_ERR_UNSUPPORTED; // the shared-memory inverse holds ts x 2ts
  static std::atomic<uint64_t> next_serial{1};
  jd.serial = next_serial.fetch_add(1);
  jd.kind = kind;
  jd.rows = p.rows;
  jd.ts   = ts;
  jd.dt   = dt;
  int *err = nullptr;
  ASGK_CUDA(cudaMalloc(&err, sizeof(int)));
  std::unique_ptr<int, decltype(&cudaFree)> err_guard(err, &cudaFree);
  ASGK_CUDA(cudaMemset(err, 0, sizeof(int)));
  // the plan's FP64 factors in the layout its indices address
  const double *vA = p.vA64;
  if (kind == ASGK_JACOBI_POINT)
  {
    size_t const b = sizeof(double) * size_t(p.rows) * ts;
    ASGK_CUDA(cudaMalloc(&jd.inv_diag, b));
    jd.device_bytes = int64_t(b);
    k_point_jacobi<<<p.rows, 128>>>(p.rows, p.d, p.n, ts, p.terms, p.mode,
                                    p.row_ptr, p.col, p.idx, vA, dt,
                                    jd.inv_diag, err);
    ASGK_LAUNCHED();
  }
  else
  {
    size_t const b = size_t(p.rows) * ts * ts;
    jd.ps16         = (ts * ts + 7) / 8 * 8;
    size_t const bh = size_t(p.rows) * jd.ps16;
    ASGK_CUDA(cudaMalloc(&jd.M64, sizeof(double) * b));
    ASGK_CUDA(cudaMalloc(&jd.M16, sizeof(__half) * bh));
    jd.device_bytes = int64_t(b * sizeof(double) + bh * sizeof(__half));
    size_t const shm = sizeof(double) * size_t(ts) * 2 * ts;
    ASGK_CUDA(cudaFuncSetAttribute(k_block_jacobi,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(shm)));
    k_block_jacobi<<<p.rows, 256, shm>>>(p.rows, p.d, p.n, ts, p.terms, p.mode,
                                         p.row_ptr, p.col, p.idx, vA, dt,
                                         jd.M64, jd.M16, jd.ps16, err);
    ASGK_LAUNCHED();
  }
  int herr = 0;
  ASGK_CUDA(cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost));
  return herr ? ASGK_ERR_BREAKDOWN : ASGK_OK;
}

int jacobi_apply(jacobi_data const &jd, bool low, double *v, double *z,
                 const double *scale_state, cudaStream_t s)
{
  int64_t const n = int64_t(jd.rows) * jd.ts;
  if (jd.kind == ASGK_JACOBI_POINT)
  {
    int const blocks = int(std::min<int64_t>((n + 255) / 256, 4096));
    k_point_apply<<<blocks, 256, 0, s>>>(n, jd.inv_diag, v, z, scale_state);
    ASGK_LAUNCHED();
    return ASGK_OK;
  }
  if (low)
  {
    if (jd.ps16 / 8 > kApply16Threads * kApply16Loads)
      return ASGK_ERR_UNSUPPORTED;
    size_t const shm = sizeof(__half) * jd.ps16 + sizeof(float) * jd.ts;
    k_block_apply16<<<jd.rows, kApply16Threads, shm, s>>>(jd.ts, jd.ps16, jd.M16, v, z,
                                                          scale_state);
  }
  else
  {
    int const threads = jd.ts <= 32 ? 32 : (jd.ts <= 64 ? 64 : 128);
    size_t const shm  = sizeof(double) * jd.ts;
    k_block_apply<double><<<jd.rows, threads, shm, s>>>(jd.rows, jd.ts, jd.M64, v, z,
                                                        scale_state);
  }
  ASGK_LAUNCHED();
  return ASGK_OK;
}

} // namespace asgk

struct asgk_jacobi
{
  asgk::jacobi_data jd;
};

int asgk_jacobi_create(asgk_jacobi **out, asgk_plan *plan, double dt, int kind)
{
  try
  {
    if (out == nullptr || plan == nullptr || !std::isfinite(dt))
      return ASGK_ERR_INVALID;
    *out = nullptr;
    std::unique_ptr<asgk_jacobi> j(new (std::nothrow) asgk_jacobi());
    if (!j)
      return ASGK_ERR_ALLOC;
    if (int rc = asgk::jacobi_build(plan->p, dt, kind, j->jd))
      return rc;
    *out = j.release();
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

void asgk_jacobi_destroy(asgk_jacobi *pc) { delete pc; }

int asgk_jacobi_apply(asgk_jacobi *pc, const double *v, double *z,
                      asgk_stream stream)
{
  try
  {
    if (pc == nullptr || v == nullptr || z == nullptr)
      return ASGK_ERR_INVALID;
    // without a scale state v is only read
    return asgk::jacobi_apply(pc->jd, false, const_cast<double *>(v), z, nullptr,
                              static_cast<cudaStream_t>(stream));
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

uint64_t asgk::jacobi_serial(const asgk_jacobi *pc) { return pc ? pc->jd.serial : 0; }

int asgk::jacobi_apply_handle(asgk_jacobi *pc, bool low, double *v, double *z,
                              const double *scale_state, cudaStream_t s)
{
  return asgk::jacobi_apply(pc->jd, low, v, z, scale_state, s);
}

int asgk_jacobi_info(asgk_jacobi *pc, int *kind, double *dt,
                     int64_t *device_bytes)
{
  try
  {
    if (pc == nullptr)
      return ASGK_ERR_INVALID;
    if (kind)
      *kind = pc->jd.kind;
    if (dt)
      *dt = pc->jd.dt;
    if (device_bytes)
      *device_bytes = pc->jd.device_bytes;
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
