// Batched Kronecker-product operator apply on sm_100a.
//
// Operator (reference: kronmult::cpu_sparse, src/device/asgard_spkronmult_cpu.cpp:84-433;
// GPU kernels src/device/asgard_spkronmult_cycle{1,2,x}.hpp):
//   y_r = beta*y_r + alpha * sum_{c in row r} sum_t (A_{t,0} (x) ... (x) A_{t,d-1}) x_c
// where every tensor has n^d entries, dimension 0 slowest, and A_{t,k} is a
// column-major n x n block.
//
// Design (differs from the reference, which runs one thread team per pair
// and atomically adds every pair's n^d results into y):
//   * one CTA owns one output cell (row) and walks that row's pair list, so y
//     is accumulated in registers and written once, coalesced, with beta,
//     alpha and the backward-Euler "+ x" term fused into the store -- no
//     atomics, no separate scaling kernel, deterministic;
//   * n = 3 fast path: a pair's 3^d tensor lives in the registers of a group
//     of 3^floor(d/2) lanes (27 for d = 6, 9 for d = 4/5, 3 for d = 2/3;
//     floor(32 / group) groups per warp, each on its own pair).  The
//     dimensions held in registers are contracted locally (9 FMAs per
//     3-fibre, no data movement); one transpose through shared memory per
//     term swaps which dimensions are in registers, and the remaining
//     dimensions are contracted locally.  Factors are uniform across a
//     group and come through the read-only path as broadcast loads.
//   * cells are visited in order of decreasing pair count (heaviest first)
//     to shorten the tail of the grid.
//   * generic path (any n, d <= 6): shared-memory stages, one output entry
//     per thread, same row ownership and fused epilogue.
#include "internal.cuh"

#include <type_traits>

namespace asgk
{
namespace
{
constexpr int ipow3(int k) { return k == 0 ? 1 : 3 * ipow3(k - 1); }

template<int D, int HL>
struct shape3
{
  static constexpr int H    = HL;                  // dimensions on lanes
  static constexpr int LG   = ipow3(H);            // lanes per group
  static constexpr int R    = ipow3(D - H);        // registers per lane
  static constexpr int TS   = ipow3(D);            // tensor size (odd)
  static constexpr int G    = 32 / LG;             // groups per warp
  static constexpr int LOWB = ipow3(D - 2 * H);    // register block below the lane dims in B
  static constexpr int BUF  = TS;                  // odd stride: conflict-free transposes
  // layout A: lane q <-> dims [0, H), register m <-> dims [H, D)
  // layout B: lane q <-> dims [H, 2H), register m <-> dims [0, H) ++ [2H, D)
  // A pair's tensor is read in layout B, dims [0, H) are contracted, one
  // transpose moves it to layout A, dims [H, D) are contracted.
  static constexpr int strideA(int k) { return ipow3(D - 1 - k); }
  static constexpr int strideB(int k) { return ipow3(H - 1 - k) * LOWB; }
  __device__ static constexpr int idxB(int q, int m)
  {
    return (m / LOWB) * ipow3(D - H) + q * LOWB + (m % LOWB);
  }
};

// lane dimensions per d: 3 x 27 registers for d = 4, 9 x 27 for d = 5,
// 27 x 27 for d = 6 (27 values per lane along every contracted fibre set)
template<int D>
struct lanes3
{
  static constexpr int value = (D <= 4) ? 1 : (D == 5 ? 2 : 3);
};

template<int B, int E, typename F>
__device__ __forceinline__ void static_for(F &&f)
{
  if constexpr (B < E)
  {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// The 9 entries of a column-major 3 x 3 factor (A(j, i) = a[j + 3 i]).
template<typename TC>
__device__ __forceinline__ void load9(const TC *__restrict__ A, TC (&a)[9])
{
#pragma unroll
  for (int i = 0; i < 9; i++)
    a[i] = __ldg(A + i);
}

// Padded block (16-byte aligned, 10 doubles or 12 floats): vector loads.
__device__ __forceinline__ void load9p(const double *__restrict__ A, double (&a)[9])
{
  const double2 *v = reinterpret_cast<const double2 *>(A);
#pragma unroll
  for (int i = 0; i < 4; i++)
  {
    double2 const t = __ldg(v + i);
    a[2 * i]        = t.x;
    a[2 * i + 1]    = t.y;
  }
  a[8] = __ldg(A + 8);
}
__device__ __forceinline__ void load9p(const float *__restrict__ A, float (&a)[9])
{
  const float4 *v = reinterpret_cast<const float4 *>(A);
  float4 const t0 = __ldg(v), t1 = __ldg(v + 1);
  a[0] = t0.x; a[1] = t0.y; a[2] = t0.z; a[3] = t0.w;
  a[4] = t1.x; a[5] = t1.y; a[6] = t1.z; a[7] = t1.w;
  a[8] = __ldg(A + 8);
}

// w <- (I (x) A (x) I) w along the register dimension with stride S:
// out_j = sum_i A(j, i) w_i.
template<int R, int S, typename TC>
__device__ __forceinline__ void contract3(TC (&w)[R], TC const (&a)[9])
{
#pragma unroll
  for (int b = 0; b < R; b++)
  {
    if ((b / S) % 3 == 0)
    {
      TC const w0 = w[b], w1 = w[b + S], w2 = w[b + 2 * S];
      w[b]         = a[0] * w0 + a[3] * w1 + a[6] * w2;
      w[b + S]     = a[1] * w0 + a[4] * w1 + a[7] * w2;
      w[b + 2 * S] = a[2] * w0 + a[5] * w1 + a[8] * w2;
    }
  }
}

// acc += (I (x) A (x) I) w along the register dimension with stride S.
template<int R, int S, typename TC>
__device__ __forceinline__ void contract3_acc(TC const (&w)[R], TC const (&a)[9],
                                              TC (&acc)[R])
{
#pragma unroll
  for (int b = 0; b < R; b++)
  {
    if ((b / S) % 3 == 0)
    {
      TC const w0 = w[b], w1 = w[b + S], w2 = w[b + 2 * S];
      acc[b]         = fma(a[6], w2, fma(a[3], w1, fma(a[0], w0, acc[b])));
      acc[b + S]     = fma(a[7], w2, fma(a[4], w1, fma(a[1], w0, acc[b + S])));
      acc[b + 2 * S] = fma(a[8], w2, fma(a[5], w1, fma(a[2], w0, acc[b + 2 * S])));
    }
  }
}

template<typename TC> struct pad3;
template<> struct pad3<double> { static constexpr int value = 10; };
template<> struct pad3<float> { static constexpr int value = 12; };

template<typename T>
__device__ __forceinline__ double to_f64(T v)
{
  return static_cast<double>(v);
}

template<int D, int HL, typename TC, typename TX, typename TY,
         index_mode MODE, bool EULER, int NW>
__global__ void __launch_bounds__(NW * 32)
    kron3_rows(int terms, const int64_t *__restrict__ row_ptr,
               const int *__restrict__ row_order, const int *__restrict__ col,
               const int *__restrict__ idx, const TC *__restrict__ vA,
               double alpha, const TX *__restrict__ x, double beta,
               TY *__restrict__ y, double ex)
{
  // conn mode: vA is the repacked [conn][d][T][pad] array
  using S = shape3<D, HL>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TC *smem = reinterpret_cast<TC *>(smem_raw);

  int const warp    = threadIdx.x >> 5;
  int const lane    = threadIdx.x & 31;
  int const g       = lane / S::LG;
  int const q       = lane - g * S::LG;
  bool const laneok = g < S::G;
  TC *buf           = smem + (warp * S::G + (laneok ? g : 0)) * S::BUF;

  int const row       = row_order[blockIdx.x];
  int64_t const pbeg  = row_ptr[row];
  int64_t const pend  = row_ptr[row + 1];
  constexpr int PAD   = pad3<TC>::value;

  TC acc[S::R];
#pragma unroll
  for (int m = 0; m < S::R; m++)
    acc[m] = TC(0);

  for (int64_t p0 = pbeg + warp * S::G; p0 < pend; p0 += NW * S::G)
  {
    int64_t const p  = p0 + g;
    bool const act   = laneok && (p < pend);
    int64_t const pc = act ? p : pbeg;

    // x in layout B: for a fixed register, the lanes of a group read
    // consecutive entries (coalesced)
    TC xb[S::R];
    {
      const TX *xs = x + int64_t(col[pc]) * S::TS;
#pragma unroll
      for (int m = 0; m < S::R; m++)
        xb[m] = act ? static_cast<TC>(xs[S::idxB(q, m)]) : TC(0);
    }
    int cn[D];
    if constexpr (MODE == index_mode::conn)
    {
#pragma unroll
      for (int k = 0; k < D; k++)
        cn[k] = __ldg(idx + pc * D + k);
    }

    for (int t = 0; t < terms; t++)
    {
      auto factor = [&](int k, TC(&a)[9]) {
        if constexpr (MODE == index_mode::conn)
          load9p(vA + ((int64_t(cn[k]) * D + k) * terms + t) * PAD, a);
        else
          load9(vA + __ldg(idx + (pc * terms + t) * D + k), a);
      };
      TC w[S::R];
#pragma unroll
      for (int m = 0; m < S::R; m++)
        w[m] = xb[m];
      // dimensions [0, H) are in registers in layout B
      static_for<0, S::H>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        TC a[9];
        factor(k, a);
        contract3<S::R, S::strideB(k)>(w, a);
      });
      // transpose to layout A through shared memory
      __syncwarp();
      if (laneok)
      {
#pragma unroll
        for (int m = 0; m < S::R; m++)
          buf[S::idxB(q, m)] = w[m];
      }
      __syncwarp();
      if (laneok)
      {
#pragma unroll
        for (int m = 0; m < S::R; m++)
          w[m] = buf[q * S::R + m];
      }
      // dimensions [H, D) are in registers in layout A; the last one
      // accumulates straight into acc
      static_for<S::H, D - 1>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        TC a[9];
        factor(k, a);
        contract3<S::R, S::strideA(k)>(w, a);
      });
      {
        TC a[9];
        factor(D - 1, a);
        if (!act)
        {
#pragma unroll
          for (int i = 0; i < 9; i++)
            a[i] = TC(0);
        }
        contract3_acc<S::R, S::strideA(D - 1)>(w, a, acc);
      }
    }
  }

  // reduce the groups' partial sums of this row and store once
  __syncwarp();
  if (laneok)
  {
#pragma unroll
    for (int m = 0; m < S::R; m++)
      buf[q * S::R + m] = acc[m];
  }
  __syncthreads();
  int64_t const base = int64_t(row) * S::TS;
  for (int i = threadIdx.x; i < S::TS; i += NW * 32)
  {
    TC s = TC(0);
#pragma unroll 4
    for (int gg = 0; gg < NW * S::G; gg++)
      s += smem[gg * S::BUF + i];
    double v = alpha * to_f64(s);
    if constexpr (EULER)
      v += ex * to_f64(x[base + i]);
    if (beta != 0.0)
      v += beta * to_f64(y[base + i]);
    y[base + i] = static_cast<TY>(v);
  }
}

// Generic (any n, d <= 6): one CTA per output cell, shared-memory stages.
template<typename TC, typename TX, typename TY, bool EULER>
__global__ void __launch_bounds__(256)
    kron_generic_rows(int d, int n, int ts, int terms, int mode,
                      const int64_t *__restrict__ row_ptr,
                      const int *__restrict__ row_order,
                      const int *__restrict__ col, const int *__restrict__ idx,
                      const TC *__restrict__ vA, double alpha,
                      const TX *__restrict__ x, double beta,
                      TY *__restrict__ y, double ex)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TC *X   = reinterpret_cast<TC *>(smem_raw);
  TC *B0  = X + ts;
  TC *B1  = B0 + ts;
  TC *ACC = B1 + ts;
  TC *F   = ACC + ts; // d * n * n factors of the current term

  int const row      = row_order[blockIdx.x];
  int64_t const pbeg = row_ptr[row];
  int64_t const pend = row_ptr[row + 1];
  int const nn       = n * n;
  int const blk      = d * terms * nn;

  for (int i = threadIdx.x; i < ts; i += blockDim.x)
    ACC[i] = TC(0);

  for (int64_t p = pbeg; p < pend; p++)
  {
    __syncthreads();
    const TX *xs = x + int64_t(col[p]) * ts;
    for (int i = threadIdx.x; i < ts; i += blockDim.x)
      X[i] = static_cast<TC>(xs[i]);
    for (int t = 0; t < terms; t++)
    {
      __syncthreads();
      for (int i = threadIdx.x; i < d * nn; i += blockDim.x)
      {
        int const k = i / nn;
        int64_t off;
        if (mode == int(index_mode::conn))
          off = int64_t(idx[p * d + k]) * blk + (t * d + k) * nn;
        else
          off = idx[(p * terms + t) * d + k];
        F[i] = vA[off + (i - k * nn)];
      }
      __syncthreads();
      const TC *src = X;
      int stride    = ts;
      for (int k = 0; k < d; k++)
      {
        stride /= n;
        TC *dst      = (k & 1) ? B1 : B0;
        const TC *A  = F + k * nn;
        for (int i = threadIdx.x; i < ts; i += blockDim.x)
        {
          int const s    = (i / stride) % n;
          int const base = i - s * stride;
          TC sum         = TC(0);
          for (int j = 0; j < n; j++)
            sum += A[s + j * n] * src[base + j * stride];
          dst[i] = sum;
        }
        __syncthreads();
        src = dst;
      }
      for (int i = threadIdx.x; i < ts; i += blockDim.x)
        ACC[i] += src[i];
    }
  }
  __syncthreads();
  int64_t const base = int64_t(row) * ts;
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
  {
    double v = alpha * static_cast<double>(ACC[i]);
    if constexpr (EULER)
      v += ex * static_cast<double>(x[base + i]);
    if (beta != 0.0)
      v += beta * static_cast<double>(y[base + i]);
    y[base + i] = static_cast<TY>(v);
  }
}

constexpr int kWarps = 4;

template<int D, typename TC, typename TX, typename TY, index_mode MODE,
         bool EULER>
int launch3(plan_data const &p, const TC *vA, double alpha, const TX *x,
            double beta, TY *y, double ex, cudaStream_t s)
{
  constexpr int HL = lanes3<D>::value;
  using S          = shape3<D, HL>;
  size_t const shm = size_t(kWarps) * S::G * S::BUF * sizeof(TC);
  auto kern        = kron3_rows<D, HL, TC, TX, TY, MODE, EULER, kWarps>;
  if constexpr (MODE == index_mode::conn)
  {
    if constexpr (std::is_same_v<TC, double>)
      vA = reinterpret_cast<const TC *>(p.vP64);
    else
      vA = reinterpret_cast<const TC *>(p.vP32);
  }
  static bool configured = false;
  if (!configured)
  {
    ASGK_CUDA(cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
    configured = true;
  }
  kern<<<p.rows, kWarps * 32, shm, s>>>(p.terms, p.row_ptr, p.row_order,
                                       p.col, p.idx, vA, alpha, x, beta, y,
                                       ex);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

template<typename TC, typename TX, typename TY, bool EULER>
int launch_generic(plan_data const &p, const TC *vA, double alpha, const TX *x,
                   double beta, TY *y, double ex, cudaStream_t s)
{
  size_t const shm =
      (size_t(4) * p.tensor + size_t(p.d) * p.n * p.n) * sizeof(TC);
  if (shm > 200 * 1024)
    return ASGK_ERR_UNSUPPORTED;
  auto kern = kron_generic_rows<TC, TX, TY, EULER>;
  ASGK_CUDA(cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
  int threads = 32;
  while (threads < p.tensor && threads < 256)
    threads *= 2;
  kern<<<p.rows, threads, shm, s>>>(p.d, p.n, p.tensor, p.terms, int(p.mode),
                                    p.row_ptr, p.row_order, p.col, p.idx, vA,
                                    alpha, x, beta, y, ex);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

template<typename TC, typename TX, typename TY, index_mode MODE, bool EULER>
int dispatch_d(plan_data const &p, const TC *vA, double alpha, const TX *x,
               double beta, TY *y, double ex, cudaStream_t s)
{
  if (p.n == 3)
  {
    switch (p.d)
    {
    case 2: return launch3<2, TC, TX, TY, MODE, EULER>(p, vA, alpha, x, beta, y, ex, s);
    case 3: return launch3<3, TC, TX, TY, MODE, EULER>(p, vA, alpha, x, beta, y, ex, s);
    case 4: return launch3<4, TC, TX, TY, MODE, EULER>(p, vA, alpha, x, beta, y, ex, s);
    case 5: return launch3<5, TC, TX, TY, MODE, EULER>(p, vA, alpha, x, beta, y, ex, s);
    case 6: return launch3<6, TC, TX, TY, MODE, EULER>(p, vA, alpha, x, beta, y, ex, s);
    default: break;
    }
  }
  return launch_generic<TC, TX, TY, EULER>(p, vA, alpha, x, beta, y, ex, s);
}

template<typename TC, typename TX, typename TY>
int dispatch(plan_data const &p, const TC *vA, double alpha, const TX *x,
             double beta, TY *y, double ex, bool euler, cudaStream_t s)
{
  if (p.mode == index_mode::conn)
    return euler ? dispatch_d<TC, TX, TY, index_mode::conn, true>(p, vA, alpha, x, beta, y, ex, s)
                 : dispatch_d<TC, TX, TY, index_mode::conn, false>(p, vA, alpha, x, beta, y, ex, s);
  return euler ? dispatch_d<TC, TX, TY, index_mode::expanded, true>(p, vA, alpha, x, beta, y, ex, s)
               : dispatch_d<TC, TX, TY, index_mode::expanded, false>(p, vA, alpha, x, beta, y, ex, s);
}

} // namespace

// y = beta*y + alpha*K*x + ex*x  (ex != 0 only for square operators)
int launch_apply(plan_data const &p, int precision, double alpha,
                 const void *x, int x_is_f32, double beta, void *y,
                 int y_is_f32, double ex, cudaStream_t s)
{
  if (p.rows == 0)
    return ASGK_OK;
  if (p.global)
  {
    if (x_is_f32 || y_is_f32)
      return ASGK_ERR_UNSUPPORTED;
    return launch_global(p, precision, alpha, static_cast<const double *>(x),
                         beta, static_cast<double *>(y), ex, s);
  }
  bool const euler = (ex != 0.0);
  if (x_is_f32 && y_is_f32)
    return dispatch<float, float, float>(p, p.vA32, alpha,
                                         static_cast<const float *>(x), beta,
                                         static_cast<float *>(y), ex, euler, s);
  if (x_is_f32 || y_is_f32)
    return ASGK_ERR_INVALID;
  if (staged_supported(p) && (precision == ASGK_FP64 || precision == ASGK_FP32))
    return launch_staged(p, precision, alpha, static_cast<const double *>(x),
                         beta, static_cast<double *>(y), ex, s);
  if (precision == ASGK_FP64)
    return dispatch<double, double, double>(p, p.vA64, alpha,
                                            static_cast<const double *>(x),
                                            beta, static_cast<double *>(y),
                                            ex, euler, s);
  if (precision == ASGK_FP32)
    return dispatch<float, double, double>(p, p.vA32, alpha,
                                           static_cast<const double *>(x),
                                           beta, static_cast<double *>(y), ex,
                                           euler, s);
  return ASGK_ERR_UNSUPPORTED;
}

} // namespace asgk
