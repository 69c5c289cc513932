// BLAS-1/2 pieces of the device-resident GMRES (FP64, HBM-bound).
//
// The reference reaches these through lib_dispatch (cuBLAS Dnrm2/Dscal/Daxpy/
// Dgemv, src/lib_dispatch.cpp:218-663); here they are plain kernels so that
// the classical Gram-Schmidt step reads the Krylov basis exactly twice (one
// multi-dot pass, one fused "w -= V h" + norm pass) and every reduction is
// deterministic: fixed grid, per-block partial sums, then an ordered sum.
#include "internal.cuh"

#include <algorithm>

namespace asgk
{
namespace
{
constexpr int kThreads = 256;

int g_sm_count = 0;

int sm_count()
{
  if (g_sm_count == 0)
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0)
      g_sm_count = 148;
  }
  return g_sm_count;
}

int grid_for(int64_t n)
{
  int64_t const want = (n + kThreads - 1) / kThreads;
  return int(std::max<int64_t>(1, std::min<int64_t>(want, 2 * int64_t(sm_count()))));
}

template<int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh)
{
  // sh: NV * 32 doubles
  int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++)
  {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  }
  if (lane == 0)
  {
#pragma unroll
    for (int i = 0; i < NV; i++)
      sh[i * 32 + warp] = v[i];
  }
  __syncthreads();
  int const nw = blockDim.x >> 5;
  if (warp == 0)
  {
#pragma unroll
    for (int i = 0; i < NV; i++)
    {
      double s = (lane < nw) ? sh[i * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
        s += __shfl_down_sync(0xffffffffu, s, o);
      v[i] = s;
    }
  }
  __syncthreads();
}

__global__ void k_fill(double *v, int64_t n, double a)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    v[i] = a;
}

__global__ void k_copy(double *__restrict__ d, const double *__restrict__ s,
                       int64_t n)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    d[i] = s[i];
}

__global__ void k_scale(double *v, int64_t n, double a)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    v[i] *= a;
}

__global__ void k_axpy(double *__restrict__ y, const double *__restrict__ x,
                       int64_t n, double a)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    y[i] += a * x[i];
}

__global__ void k_xpby(double *__restrict__ y, const double *__restrict__ x,
                       int64_t n, double b)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    y[i] = x[i] + b * y[i];
}

// part[b*k + j] = sum over row chunk b of V[r, j] * w[r]; block (b, g)
// takes the columns 8g .. 8g+7 of chunk b (one block reduction each)
constexpr int kDotCols = 8;
__global__ void __launch_bounds__(kThreads)
    k_multidot(const double *__restrict__ V, int64_t ldv, int k,
               const double *__restrict__ w, int64_t n,
               double *__restrict__ part)
{
  __shared__ double sh[kDotCols * 32];
  int64_t const chunk = (n + gridDim.x - 1) / gridDim.x;
  int64_t const beg   = blockIdx.x * chunk;
  int64_t const end   = min(n, beg + chunk);
  int const j0        = blockIdx.y * kDotCols;
  int const nj        = min(kDotCols, k - j0);
  double a[kDotCols];
#pragma unroll
  for (int j = 0; j < kDotCols; j++)
    a[j] = 0.0;
  const double *Vj = V + int64_t(j0) * ldv;
  for (int64_t r = beg + threadIdx.x; r < end; r += blockDim.x)
  {
    double const wr = w[r];
#pragma unroll
    for (int j = 0; j < kDotCols; j++)
      if (j < nj)
        a[j] = fma(Vj[r + j * ldv], wr, a[j]);
  }
  block_sum<kDotCols>(a, sh);
  if (threadIdx.x == 0)
    for (int j = 0; j < nj; j++)
      part[int64_t(blockIdx.x) * k + j0 + j] = a[j];
}

__global__ void k_reduce_parts(const double *__restrict__ part, int blocks,
                               int k, double *__restrict__ out)
{
  __shared__ double sh[32];
  int const j = blockIdx.x;
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < blocks; b += blockDim.x)
    v[0] += part[int64_t(b) * k + j];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0)
    out[j] = v[0];
}

// w -= V[:, :k] h ; part[b] = sum of w^2 over block b's rows.  Four
// independent partial sums per row keep four basis loads in flight.
__device__ __forceinline__ double dot_row(const double *__restrict__ V,
                                          int64_t ldv, int k, int64_t r,
                                          const double *hs)
{
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int j = 0;
  for (; j + 4 <= k; j += 4)
  {
    s0 = fma(V[r + j * ldv], hs[j], s0);
    s1 = fma(V[r + (j + 1) * ldv], hs[j + 1], s1);
    s2 = fma(V[r + (j + 2) * ldv], hs[j + 2], s2);
    s3 = fma(V[r + (j + 3) * ldv], hs[j + 3], s3);
  }
  for (; j < k; j++)
    s0 = fma(V[r + j * ldv], hs[j], s0);
  return (s0 + s1) + (s2 + s3);
}

__global__ void __launch_bounds__(kThreads)
    k_update_norm(const double *__restrict__ V, int64_t ldv, int k,
                  const double *__restrict__ h, double *__restrict__ w,
                  int64_t n, double *__restrict__ part)
{
  extern __shared__ double hs[];
  __shared__ double sh[32];
  for (int j = threadIdx.x; j < k; j += blockDim.x)
    hs[j] = h[j];
  __syncthreads();
  int64_t const chunk = (n + gridDim.x - 1) / gridDim.x;
  int64_t const beg   = blockIdx.x * chunk;
  int64_t const end   = min(n, beg + chunk);
  double v[1]         = {0.0};
  for (int64_t r = beg + threadIdx.x; r < end; r += blockDim.x)
  {
    double const wr = w[r] - dot_row(V, ldv, k, r, hs);
    w[r]            = wr;
    v[0] += wr * wr;
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0)
    part[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(kThreads)
    k_norm2(const double *__restrict__ x, int64_t n, double *__restrict__ part)
{
  __shared__ double sh[32];
  int64_t const chunk = (n + gridDim.x - 1) / gridDim.x;
  int64_t const beg   = blockIdx.x * chunk;
  int64_t const end   = min(n, beg + chunk);
  double v[1]         = {0.0};
  for (int64_t r = beg + threadIdx.x; r < end; r += blockDim.x)
    v[0] += x[r] * x[r];
  block_sum<1>(v, sh);
  if (threadIdx.x == 0)
    part[blockIdx.x] = v[0];
}

// x += V[:, :k] y
__global__ void __launch_bounds__(kThreads)
    k_gemv_add(const double *__restrict__ V, int64_t ldv, int k,
               const double *__restrict__ y, double *__restrict__ x, int64_t n)
{
  extern __shared__ double ys[];
  for (int j = threadIdx.x; j < k; j += blockDim.x)
    ys[j] = y[j];
  __syncthreads();
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x)
    x[r] += dot_row(V, ldv, k, r, ys);
}

} // namespace

int max_reduction_blocks() { return 2 * sm_count(); }

int launch_fill(double *v, int64_t n, double a, cudaStream_t s)
{
  k_fill<<<grid_for(n), kThreads, 0, s>>>(v, n, a);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_copy(double *d, const double *src, int64_t n, cudaStream_t s)
{
  k_copy<<<grid_for(n), kThreads, 0, s>>>(d, src, n);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_scale(double *v, int64_t n, double a, cudaStream_t s)
{
  k_scale<<<grid_for(n), kThreads, 0, s>>>(v, n, a);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_axpy(double *y, const double *x, int64_t n, double a, cudaStream_t s)
{
  k_axpy<<<grid_for(n), kThreads, 0, s>>>(y, x, n, a);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_xpby(double *y, const double *x, int64_t n, double b, cudaStream_t s)
{
  k_xpby<<<grid_for(n), kThreads, 0, s>>>(y, x, n, b);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_multidot(const double *V, int64_t ldv, int k, const double *w,
                    int64_t n, double *part, int *blocks, cudaStream_t s)
{
  int const g = grid_for(n);
  dim3 const grid(g, (k + kDotCols - 1) / kDotCols);
  k_multidot<<<grid, kThreads, 0, s>>>(V, ldv, k, w, n, part);
  ASGK_LAUNCHED();
  *blocks = g;
  return ASGK_OK;
}

int launch_reduce_parts(const double *part, int blocks, int k, double *out,
                        cudaStream_t s)
{
  k_reduce_parts<<<k, kThreads, 0, s>>>(part, blocks, k, out);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_update_norm(const double *V, int64_t ldv, int k, const double *h,
                       double *w, int64_t n, double *part, int *blocks,
                       cudaStream_t s)
{
  int const g = grid_for(n);
  k_update_norm<<<g, kThreads, sizeof(double) * std::max(k, 1), s>>>(
      V, ldv, k, h, w, n, part);
  ASGK_LAUNCHED();
  *blocks = g;
  return ASGK_OK;
}

int launch_norm2(const double *v, int64_t n, double *part, int *blocks,
                 cudaStream_t s)
{
  int const g = grid_for(n);
  k_norm2<<<g, kThreads, 0, s>>>(v, n, part);
  ASGK_LAUNCHED();
  *blocks = g;
  return ASGK_OK;
}

int launch_gemv_add(const double *V, int64_t ldv, int k, const double *y,
                    double *x, int64_t n, cudaStream_t s)
{
  k_gemv_add<<<grid_for(n), kThreads, sizeof(double) * std::max(k, 1), s>>>(
      V, ldv, k, y, x, n);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

} // namespace asgk
