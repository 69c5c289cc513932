// BLAS-1/2 pieces of the device-resident GMRES (FP64, HBM-bound).
//
// The reference reaches these through lib_dispatch (cuBLAS Dnrm2/Dscal/Daxpy/
// Dgemv, src/lib_dispatch.cpp:218-663); here they are plain kernels so that
// the classical Gram-Schmidt step reads the Krylov basis exactly twice (one
// multi-dot pass, one fused "w -= V h" + norm pass) and every reduction is
// deterministic: fixed grid, per-block partial sums, then an ordered sum.
#include "gmres_device.cuh"

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

// x += V[:, :k] y; VEC = 2 takes two rows per 16-byte load, with each row's
// sum in the order of dot_row (four chains by column mod 4), so both forms
// give the same bits
template<int VEC>
__global__ void __launch_bounds__(kThreads)
    k_gemv_add(const double *__restrict__ V, int64_t ldv, int k,
               const double *__restrict__ y, double *__restrict__ x, int64_t n)
{
  extern __shared__ double ys[];
  for (int j = threadIdx.x; j < k; j += blockDim.x)
    ys[j] = y[j];
  __syncthreads();
  if constexpr (VEC == 1)
  {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
         r += int64_t(gridDim.x) * blockDim.x)
      x[r] += dot_row(V, ldv, k, r, ys);
  }
  else
  {
    const double2 *V2 = reinterpret_cast<const double2 *>(V);
    int64_t const ld2 = ldv / 2;
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n / 2;
         r += int64_t(gridDim.x) * blockDim.x)
    {
      double a[4] = {0.0, 0.0, 0.0, 0.0}, b[4] = {0.0, 0.0, 0.0, 0.0};
      int j = 0;
      for (; j + 4 <= k; j += 4)
      {
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
          double2 const v = V2[r + (j + q) * ld2];
          a[q]            = fma(v.x, ys[j + q], a[q]);
          b[q]            = fma(v.y, ys[j + q], b[q]);
        }
      }
      for (; j < k; j++)
      {
        double2 const v = V2[r + j * ld2];
        a[0]            = fma(v.x, ys[j], a[0]);
        b[0]            = fma(v.y, ys[j], b[0]);
      }
      double2 *x2 = reinterpret_cast<double2 *>(x);
      double2 t   = x2[r];
      t.x += (a[0] + a[1]) + (a[2] + a[3]);
      t.y += (b[0] + b[1]) + (b[2] + b[3]);
      x2[r] = t;
    }
  }
}

// ---- Gram-Schmidt kernels that finish their own reductions -------------
//
// Each block writes its partial sums, then the last block to finish (an
// atomic ticket; the ticket is reset for the next launch) adds them in block
// order -- the same fixed order whichever block ends last, so results are
// deterministic -- and writes the totals.  This saves the separate
// reduction launch after every pass.  VEC = 2 reads two rows per 16-byte
// load (n and the leading dimension even, 16-byte aligned vectors).

// out[c0 + c] = sum_b part[b*stride + c0 + c], c < nc: one warp per column,
// lanes over the blocks in a fixed assignment, a fixed shuffle tree
__device__ __forceinline__ void ordered_column_sums(const double *part, int nb,
                                                    int stride, int c0, int nc,
                                                    double *out)
{
  int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = warp; c < nc; c += blockDim.x >> 5)
  {
    double s = 0.0;
    for (int b = lane; b < nb; b += 32)
      s += __ldcg(part + int64_t(b) * stride + c0 + c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0)
      out[c0 + c] = s;
  }
}

// thread 0 publishes this block's partials (already in part) and takes a
// ticket; true in every thread of the block that finished last
__device__ __forceinline__ bool last_block(unsigned *ticket, unsigned nblocks)
{
  __shared__ unsigned s_last;
  if (threadIdx.x == 0)
  {
    __threadfence();
    s_last = (atomicAdd(ticket, 1u) == nblocks - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (s_last)
    __threadfence();
  return s_last != 0;
}

// The end of an update pass: this block's partial of ||w||^2, the ordered
// total from the last block, then (ga.state set: a recorded GMRES step) the
// step's Givens update: earlier rotations staged in shared memory after the
// k coefficients, then one thread (the serial part touches shared memory
// only).
__device__ __forceinline__ void finish_update(double (&v)[1], double *sh,
                                              double *hs, int k, double *part,
                                              unsigned *ticket, double *out,
                                              givens_args const &ga)
{
  block_sum<1>(v, sh);
  if (threadIdx.x == 0)
    part[blockIdx.x] = v[0];
  if (!last_block(ticket, gridDim.x))
    return;
  ordered_column_sums(part, gridDim.x, 1, 0, 1, out);
  if (threadIdx.x == 0)
    *ticket = 0u;
  if (ga.state == nullptr)
    return;
  double *csn    = hs + k;                     // cosines, sines: 2*(restart+1)
  double *coeffs = csn + 2 * (ga.restart + 1); // k
  const double *cs_g = ga.state + kStateHead + ga.restart + 1;
  for (int j = threadIdx.x; j < 2 * (ga.restart + 1); j += blockDim.x)
    csn[j] = (j % (ga.restart + 1) < ga.step) ? cs_g[j] : 0.0;
  __syncthreads();
  if (threadIdx.x == 0)
    givens_step(ga, hs, *out, coeffs, csn);
}

template<int VEC> struct vload;
template<> struct vload<1>
{
  using T = double;
};
template<> struct vload<2>
{
  using T = double2;
};

// h[j] = V[:, j] . w for j < k; grid (row chunks, column groups of 8)
template<int VEC>
__global__ void __launch_bounds__(kThreads)
    k_multidot_h(const double *__restrict__ V, int64_t ldv, int k,
                 const double *__restrict__ w, int64_t n,
                 double *__restrict__ part, unsigned *__restrict__ tickets,
                 double *__restrict__ h, const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  using T = typename vload<VEC>::T;
  __shared__ double sh[kDotCols * 32];
  int64_t const nu    = n / VEC;
  int64_t const chunk = (nu + gridDim.x - 1) / gridDim.x;
  int64_t const beg   = blockIdx.x * chunk;
  int64_t const end   = min(nu, beg + chunk);
  int const j0        = blockIdx.y * kDotCols;
  int const nj        = min(kDotCols, k - j0);
  int64_t const ldu   = ldv / VEC;
  double a[kDotCols];
#pragma unroll
  for (int j = 0; j < kDotCols; j++)
    a[j] = 0.0;
  const T *Vj = reinterpret_cast<const T *>(V + int64_t(j0) * ldv);
  const T *wu = reinterpret_cast<const T *>(w);
  for (int64_t r = beg + threadIdx.x; r < end; r += blockDim.x)
  {
    T const wr = wu[r];
#pragma unroll
    for (int j = 0; j < kDotCols; j++)
      if (j < nj)
      {
        T const v = Vj[r + j * ldu];
        if constexpr (VEC == 1)
          a[j] = fma(v, wr, a[j]);
        else
          a[j] = fma(v.y, wr.y, fma(v.x, wr.x, a[j]));
      }
  }
  block_sum<kDotCols>(a, sh);
  if (threadIdx.x == 0)
    for (int j = 0; j < nj; j++)
      part[int64_t(blockIdx.x) * k + j0 + j] = a[j];
  if (!last_block(tickets + blockIdx.y, gridDim.x))
    return;
  ordered_column_sums(part, gridDim.x, k, j0, nj, h);
  if (threadIdx.x == 0)
    tickets[blockIdx.y] = 0u;
}

// w -= V[:, :k] h;  *out = ||w||^2; with ga.state set (a recorded GMRES
// step), the last block then performs the step's Givens update.  Dynamic
// shared memory: k doubles, plus 3*(restart+1) with a Givens update.
template<int VEC>
__global__ void __launch_bounds__(kThreads)
    k_update_norm_h(const double *__restrict__ V, int64_t ldv, int k,
                    const double *__restrict__ h, double *__restrict__ w,
                    int64_t n, double *__restrict__ part,
                    unsigned *__restrict__ ticket, double *__restrict__ out,
                    givens_args ga, const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  using T = typename vload<VEC>::T;
  extern __shared__ double hs[];
  __shared__ double sh[32];
  for (int j = threadIdx.x; j < k; j += blockDim.x)
    hs[j] = h[j];
  __syncthreads();
  int64_t const nu    = n / VEC;
  int64_t const chunk = (nu + gridDim.x - 1) / gridDim.x;
  int64_t const beg   = blockIdx.x * chunk;
  int64_t const end   = min(nu, beg + chunk);
  int64_t const ldu   = ldv / VEC;
  const T *Vu = reinterpret_cast<const T *>(V);
  T *wu       = reinterpret_cast<T *>(w);
  double v[1] = {0.0};
  for (int64_t r = beg + threadIdx.x; r < end; r += blockDim.x)
  {
    if constexpr (VEC == 1)
    {
      double const wr = wu[r] - dot_row(V, ldv, k, r, hs);
      wu[r]           = wr;
      v[0] += wr * wr;
    }
    else
    {
      // two rows, eight basis loads in flight (four partial sums per row)
      double x0 = 0.0, x1 = 0.0, x2 = 0.0, x3 = 0.0;
      double y0 = 0.0, y1 = 0.0, y2 = 0.0, y3 = 0.0;
      int j = 0;
      for (; j + 8 <= k; j += 8)
      {
        T u[8];
#pragma unroll
        for (int q = 0; q < 8; q++)
          u[q] = Vu[r + (j + q) * ldu];
#pragma unroll
        for (int q = 0; q < 8; q += 4)
        {
          x0 = fma(u[q].x, hs[j + q], x0);
          y0 = fma(u[q].y, hs[j + q], y0);
          x1 = fma(u[q + 1].x, hs[j + q + 1], x1);
          y1 = fma(u[q + 1].y, hs[j + q + 1], y1);
          x2 = fma(u[q + 2].x, hs[j + q + 2], x2);
          y2 = fma(u[q + 2].y, hs[j + q + 2], y2);
          x3 = fma(u[q + 3].x, hs[j + q + 3], x3);
          y3 = fma(u[q + 3].y, hs[j + q + 3], y3);
        }
      }
      for (; j + 4 <= k; j += 4)
      {
        T const a = Vu[r + j * ldu], b = Vu[r + (j + 1) * ldu];
        T const c = Vu[r + (j + 2) * ldu], d = Vu[r + (j + 3) * ldu];
        x0 = fma(a.x, hs[j], x0);
        y0 = fma(a.y, hs[j], y0);
        x1 = fma(b.x, hs[j + 1], x1);
        y1 = fma(b.y, hs[j + 1], y1);
        x2 = fma(c.x, hs[j + 2], x2);
        y2 = fma(c.y, hs[j + 2], y2);
        x3 = fma(d.x, hs[j + 3], x3);
        y3 = fma(d.y, hs[j + 3], y3);
      }
      for (; j < k; j++)
      {
        T const a = Vu[r + j * ldu];
        x0 = fma(a.x, hs[j], x0);
        y0 = fma(a.y, hs[j], y0);
      }
      T wr = wu[r];
      wr.x -= (x0 + x1) + (x2 + x3);
      wr.y -= (y0 + y1) + (y2 + y3);
      wu[r] = wr;
      v[0] += wr.x * wr.x + wr.y * wr.y;
    }
  }
  finish_update(v, sh, hs, k, part, ticket, out, ga);
}

// ---- the same two passes over an FP32 copy of the basis -----------------
//
// In the FP32 inner solves of iterative refinement the basis columns used
// by Gram-Schmidt are stored in FP32 beside the FP64 ones (which the
// operator and the solution update keep reading): the two passes move half
// the bytes, and a 50-column basis of the benchmark sizes stays in L2.  w,
// h and all sums stay FP64.  VEC = 4 reads four rows per 16-byte load (n
// and the leading dimension multiples of 4, 16-byte aligned vectors).

template<int VEC> struct fload;
template<> struct fload<1>
{
  using T = float;
};
template<> struct fload<4>
{
  using T = float4;
};
__device__ __forceinline__ double fcomp(float a, int) { return double(a); }
__device__ __forceinline__ double fcomp(float4 const &a, int e)
{
  return double(e == 0 ? a.x : e == 1 ? a.y : e == 2 ? a.z : a.w);
}

// rows VEC*r .. VEC*r + VEC - 1 of w
template<int VEC>
__device__ __forceinline__ void load_rows(const double *w, int64_t r, double (&o)[VEC])
{
  if constexpr (VEC == 1)
    o[0] = w[r];
  else
  {
    const double2 *p = reinterpret_cast<const double2 *>(w) + r * (VEC / 2);
#pragma unroll
    for (int q = 0; q < VEC / 2; q++)
    {
      double2 const t = p[q];
      o[2 * q]        = t.x;
      o[2 * q + 1]    = t.y;
    }
  }
}
template<int VEC>
__device__ __forceinline__ void store_rows(double *w, int64_t r, double const (&o)[VEC])
{
  if constexpr (VEC == 1)
    w[r] = o[0];
  else
  {
    double2 *p = reinterpret_cast<double2 *>(w) + r * (VEC / 2);
#pragma unroll
    for (int q = 0; q < VEC / 2; q++)
      p[q] = make_double2(o[2 * q], o[2 * q + 1]);
  }
}

// h[j] = V[:, j] . w for j < k (V FP32); grid (row chunks, column groups)
template<int VEC>
__global__ void __launch_bounds__(kThreads)
    k_multidot_f(const float *__restrict__ V, int64_t ldv, int k,
                 const double *__restrict__ w, int64_t n,
                 double *__restrict__ part, unsigned *__restrict__ tickets,
                 double *__restrict__ h, const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  using T = typename fload<VEC>::T;
  __shared__ double sh[kDotCols * 32];
  int64_t const nu    = n / VEC;
  int64_t const chunk = (nu + gridDim.x - 1) / gridDim.x;
  int64_t const beg   = blockIdx.x * chunk;
  int64_t const end   = min(nu, beg + chunk);
  int const j0        = blockIdx.y * kDotCols;
  int const nj        = min(kDotCols, k - j0);
  int64_t const ldu   = ldv / VEC;
  double a[kDotCols];
#pragma unroll
  for (int j = 0; j < kDotCols; j++)
    a[j] = 0.0;
  const T *Vj = reinterpret_cast<const T *>(V + int64_t(j0) * ldv);
  for (int64_t r = beg + threadIdx.x; r < end; r += blockDim.x)
  {
    double wr[VEC];
    load_rows<VEC>(w, r, wr);
#pragma unroll
    for (int j = 0; j < kDotCols; j++)
      if (j < nj)
      {
        T const v = Vj[r + j * ldu];
#pragma unroll
        for (int e = 0; e < VEC; e++)
          a[j] = fma(fcomp(v, e), wr[e], a[j]);
      }
  }
  block_sum<kDotCols>(a, sh);
  if (threadIdx.x == 0)
    for (int j = 0; j < nj; j++)
      part[int64_t(blockIdx.x) * k + j0 + j] = a[j];
  if (!last_block(tickets + blockIdx.y, gridDim.x))
    return;
  ordered_column_sums(part, gridDim.x, k, j0, nj, h);
  if (threadIdx.x == 0)
    tickets[blockIdx.y] = 0u;
}

// w -= V[:, :k] h (V FP32); *out = ||w||^2; the Givens update of a recorded
// step as in k_update_norm_h
template<int VEC>
__global__ void __launch_bounds__(kThreads)
    k_update_norm_f(const float *__restrict__ V, int64_t ldv, int k,
                    const double *__restrict__ h, double *__restrict__ w,
                    int64_t n, double *__restrict__ part,
                    unsigned *__restrict__ ticket, double *__restrict__ out,
                    givens_args ga, const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  using T = typename fload<VEC>::T;
  extern __shared__ double hs[];
  __shared__ double sh[32];
  for (int j = threadIdx.x; j < k; j += blockDim.x)
    hs[j] = h[j];
  __syncthreads();
  int64_t const nu    = n / VEC;
  int64_t const chunk = (nu + gridDim.x - 1) / gridDim.x;
  int64_t const beg   = blockIdx.x * chunk;
  int64_t const end   = min(nu, beg + chunk);
  int64_t const ldu   = ldv / VEC;
  const T *Vu         = reinterpret_cast<const T *>(V);
  double v[1]         = {0.0};
  for (int64_t r = beg + threadIdx.x; r < end; r += blockDim.x)
  {
    // eight basis loads in flight, four partial sums per row
    double acc[4][VEC];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int e = 0; e < VEC; e++)
        acc[q][e] = 0.0;
    int j = 0;
    for (; j + 8 <= k; j += 8)
    {
      T u[8];
#pragma unroll
      for (int q = 0; q < 8; q++)
        u[q] = Vu[r + (j + q) * ldu];
#pragma unroll
      for (int q = 0; q < 8; q++)
#pragma unroll
        for (int e = 0; e < VEC; e++)
          acc[q & 3][e] = fma(fcomp(u[q], e), hs[j + q], acc[q & 3][e]);
    }
    for (; j < k; j++)
    {
      T const u = Vu[r + j * ldu];
#pragma unroll
      for (int e = 0; e < VEC; e++)
        acc[0][e] = fma(fcomp(u, e), hs[j], acc[0][e]);
    }
    double wr[VEC];
    load_rows<VEC>(w, r, wr);
#pragma unroll
    for (int e = 0; e < VEC; e++)
    {
      wr[e] -= (acc[0][e] + acc[1][e]) + (acc[2][e] + acc[3][e]);
      v[0] += wr[e] * wr[e];
    }
    store_rows<VEC>(w, r, wr);
  }
  finish_update(v, sh, hs, k, part, ticket, out, ga);
}

// w *= f and vf = FP32(w), f = state[1] (the 1/||w|| of a recorded step) or
// scale: a new basis vector normalised, with its FP32 copy
template<int VEC>
__global__ void k_store_basis(double *__restrict__ w, float *__restrict__ vf,
                              int64_t n, const double *__restrict__ state,
                              double scale, const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  double const f = state ? state[1] : scale;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n / VEC;
       r += int64_t(gridDim.x) * blockDim.x)
  {
    double x[VEC];
    load_rows<VEC>(w, r, x);
#pragma unroll
    for (int e = 0; e < VEC; e++)
      x[e] *= f;
    store_rows<VEC>(w, r, x);
    if constexpr (VEC == 1)
      vf[r] = float(x[0]);
    else
      reinterpret_cast<float2 *>(vf)[r] = make_float2(float(x[0]), float(x[1]));
  }
}

// *out = ||x||^2
__global__ void __launch_bounds__(kThreads)
    k_norm2_h(const double *__restrict__ x, int64_t n,
              double *__restrict__ part, unsigned *__restrict__ ticket,
              double *__restrict__ out)
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
  if (!last_block(ticket, gridDim.x))
    return;
  ordered_column_sums(part, gridDim.x, 1, 0, 1, out);
  if (threadIdx.x == 0)
    *ticket = 0u;
}

// blocks of the self-reducing passes: up to eight per SM (full occupancy at
// 256 threads), so enough basis loads are in flight; the multi-dot shares
// them among its column groups
int grid_wide(int64_t n, int groups = 1)
{
  int64_t const want = (n + kThreads - 1) / kThreads;
  int64_t const cap  = std::max<int64_t>(2 * sm_count(), 8 * int64_t(sm_count()) / groups);
  return int(std::max<int64_t>(1, std::min(want, cap)));
}

// v *= a[1] (the 1/||w|| a recorded GMRES step leaves in its device state)
__global__ void k_scale_by(double *v, int64_t n, const double *__restrict__ a,
                           const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  double const f = a[1];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    v[i] *= f;
}

bool vec2_ok(const double *a, int64_t ld, const double *b)
{
  return (ld % 2 == 0) && (reinterpret_cast<uintptr_t>(a) % 16 == 0) &&
         (reinterpret_cast<uintptr_t>(b) % 16 == 0);
}

bool vec4_ok(const float *a, int64_t ld, const double *b, int64_t n)
{
  return (n % 4 == 0) && (ld % 4 == 0) && (reinterpret_cast<uintptr_t>(a) % 16 == 0) &&
         (reinterpret_cast<uintptr_t>(b) % 16 == 0);
}

} // namespace

int max_reduction_blocks() { return 2 * sm_count(); }
int max_reduction_blocks_wide() { return 8 * sm_count(); }

int launch_multidot_h(const double *V, int64_t ldv, int k, const double *w,
                      int64_t n, double *part, unsigned *tickets, double *h,
                      cudaStream_t s)
{
  int const groups = (k + kDotCols - 1) / kDotCols;
  // one block per SM and column group (measured: more row blocks lengthen
  // the final sums more than they shorten the pass)
  dim3 const grid(std::min(grid_for(n), sm_count()), groups);
  if (vec2_ok(V, ldv, w) && n % 2 == 0)
    k_multidot_h<2><<<grid, kThreads, 0, s>>>(V, ldv, k, w, n, part, tickets, h, g_gate);
  else
    k_multidot_h<1><<<grid, kThreads, 0, s>>>(V, ldv, k, w, n, part, tickets, h, g_gate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_update_norm_h(const double *V, int64_t ldv, int k, const double *h,
                         double *w, int64_t n, double *part, unsigned *ticket,
                         double *out, cudaStream_t s, givens_args const *ga)
{
  int const g        = grid_for(n); // two blocks per SM (measured best)
  givens_args const a = ga ? *ga : givens_args{};
  size_t const shm   = sizeof(double) *
                     (std::max(k, 1) + (ga ? 3 * int64_t(a.restart + 1) : 0));
  if (vec2_ok(V, ldv, w) && n % 2 == 0)
    k_update_norm_h<2><<<g, kThreads, shm, s>>>(V, ldv, k, h, w, n, part, ticket, out, a,
                                                g_gate);
  else
    k_update_norm_h<1><<<g, kThreads, shm, s>>>(V, ldv, k, h, w, n, part, ticket, out, a,
                                                g_gate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_multidot_hf(const float *V, int64_t ldv, int k, const double *w,
                       int64_t n, double *part, unsigned *tickets, double *h,
                       cudaStream_t s)
{
  int const groups = (k + kDotCols - 1) / kDotCols;
  // four blocks per SM per column group (d=6, level 7: 1 -> 4 per SM took
  // the method solve from 24.8 to 23.2 ms; the partial sums stay within the
  // workspace's 8 * SMs rows)
  dim3 const grid(std::min<int64_t>((n + kThreads - 1) / kThreads, 4 * int64_t(sm_count())), groups);
  if (vec4_ok(V, ldv, w, n))
    k_multidot_f<4><<<grid, kThreads, 0, s>>>(V, ldv, k, w, n, part, tickets, h, g_gate);
  else
    k_multidot_f<1><<<grid, kThreads, 0, s>>>(V, ldv, k, w, n, part, tickets, h, g_gate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_update_norm_hf(const float *V, int64_t ldv, int k, const double *h,
                          double *w, int64_t n, double *part, unsigned *ticket,
                          double *out, cudaStream_t s, givens_args const *ga)
{
  // every resident block (eight per SM): more basis loads in flight
  int const g        = int(std::min<int64_t>((n + kThreads - 1) / kThreads, 8 * int64_t(sm_count())));
  givens_args const a = ga ? *ga : givens_args{};
  size_t const shm   = sizeof(double) *
                     (std::max(k, 1) + (ga ? 3 * int64_t(a.restart + 1) : 0));
  if (vec4_ok(V, ldv, w, n))
    k_update_norm_f<4><<<g, kThreads, shm, s>>>(V, ldv, k, h, w, n, part, ticket, out, a,
                                                g_gate);
  else
    k_update_norm_f<1><<<g, kThreads, shm, s>>>(V, ldv, k, h, w, n, part, ticket, out, a,
                                                g_gate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_store_basis(double *w, float *vf, int64_t n, const double *state,
                       double scale, cudaStream_t s)
{
  bool const v2 = (n % 2 == 0) && (reinterpret_cast<uintptr_t>(w) % 16 == 0) &&
                  (reinterpret_cast<uintptr_t>(vf) % 8 == 0);
  if (v2)
    k_store_basis<2><<<grid_wide(n / 2), kThreads, 0, s>>>(w, vf, n, state, scale, g_gate);
  else
    k_store_basis<1><<<grid_wide(n), kThreads, 0, s>>>(w, vf, n, state, scale, g_gate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_scale_by(double *v, int64_t n, const double *state, cudaStream_t s)
{
  k_scale_by<<<grid_wide(n), kThreads, 0, s>>>(v, n, state, g_gate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_norm2_h(const double *v, int64_t n, double *part, unsigned *ticket,
                   double *out, cudaStream_t s)
{
  k_norm2_h<<<grid_wide(n), kThreads, 0, s>>>(v, n, part, ticket, out);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_fill(double *v, int64_t n, double a, cudaStream_t s)
{
  k_fill<<<grid_wide(n), kThreads, 0, s>>>(v, n, a);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_copy(double *d, const double *src, int64_t n, cudaStream_t s)
{
  k_copy<<<grid_wide(n), kThreads, 0, s>>>(d, src, n);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_scale(double *v, int64_t n, double a, cudaStream_t s)
{
  k_scale<<<grid_wide(n), kThreads, 0, s>>>(v, n, a);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_axpy(double *y, const double *x, int64_t n, double a, cudaStream_t s)
{
  k_axpy<<<grid_wide(n), kThreads, 0, s>>>(y, x, n, a);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

int launch_xpby(double *y, const double *x, int64_t n, double b, cudaStream_t s)
{
  k_xpby<<<grid_wide(n), kThreads, 0, s>>>(y, x, n, b);
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
  size_t const sh = sizeof(double) * std::max(k, 1);
  if (n % 2 == 0 && vec2_ok(V, ldv, x))
    k_gemv_add<2><<<grid_wide(n / 2), kThreads, sh, s>>>(V, ldv, k, y, x, n);
  else
    k_gemv_add<1><<<grid_wide(n), kThreads, sh, s>>>(V, ldv, k, y, x, n);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

} // namespace asgk
