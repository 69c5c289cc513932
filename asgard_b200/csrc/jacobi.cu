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
// kron: the same block inverse for global plans whose terms act in one
//   dimension each, where a cell's diagonal block is the Kronecker sum
//   (1 - dt n_identity) I - dt sum_k (I (x) B_k (x) I) of its 3x3 self
//   blocks B_k: with B_k = V_k diag(lambda_k) V_k^-1 (eigendecompositions on
//   the host, one per 1D cell and dimension) the inverse is
//   (x)_k V_k diag(1 / mu) (x)_k V_k^-1, mu = (1 - dt n_identity)
//   - dt sum_k lambda_k,i_k, applied in 2d complex contractions per cell
//   from a few hundred bytes of tables instead of the n^d x n^d inverse.
#include "internal.cuh"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <new>
#include <vector>

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
                              const double *__restrict__ scale_state,
                              float *__restrict__ vcopy,
                              const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
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
      if (vcopy)
        vcopy[int64_t(row) * ts + i] = float(vv);
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
                    const double *__restrict__ scale_state,
                    float *__restrict__ vcopy, const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
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
      if (vcopy)
        vcopy[int64_t(row) * ts + i] = static_cast<float>(vv);
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
                              const double *__restrict__ scale_state,
                              float *__restrict__ vcopy,
                              const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  double const f = scale_state ? scale_state[1] : 1.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    double vv = v[i];
    if (scale_state)
    {
      vv   = vv * f;
      v[i] = vv;
      if (vcopy)
        vcopy[i] = float(vv);
    }
    z[i] = vv * inv_diag[i];
  }
}

// ---- Kronecker-sum block inverse -------------------------------------------
// Table entry of one (1D cell, dimension): V (3x3), W = V^-1 (3x3), column-
// major, then the 3 eigenvalues; complex values as (re, im) pairs.
constexpr int kKronTab = 42;

constexpr int ipow3j(int k) { return k == 0 ? 1 : 3 * ipow3j(k - 1); }

// One warp per cell: u = v (scaled by scale_state[1] in place first when
// given, and then also written rounded to FP32 into vcopy when given), u <- (I (x) W_k (x) I) u for every k, u_i /= mu_i,
// u <- (I (x) V_k (x) I) u for every k, z = Re u.  The cell's D tables are
// staged in shared memory and the loops over dimensions unrolled; a stage
// gives each lane whole fibres (three loads, nine complex multiply-adds,
// three stores).  Shared memory per warp: 2 buffers x (re, im) x 3^D values,
// then D tables.
template<typename R, int D, int WPC>
__global__ void __launch_bounds__(WPC * 32)
    k_kron_apply(int rows, const int *__restrict__ kself,
                 const R *__restrict__ tab, double shift, double dt,
                 double *__restrict__ v, double *__restrict__ z,
                 const double *__restrict__ scale_state,
                 float *__restrict__ vcopy, const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  constexpr int TS  = ipow3j(D);
  constexpr int PER = (TS + 31) / 32;
  constexpr int WS  = 4 * TS + D * kKronTab; // per-warp shared values
  // up to four entries per lane keep their digits in registers; more (d >= 5)
  // divide by the compile-time strides instead
  constexpr bool KEEP = PER <= 4;
  constexpr int PD    = KEEP ? PER : 1;
  extern __shared__ __align__(16) unsigned char kron_smem[];
  int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int const c    = blockIdx.x * WPC + warp;
  if (c >= rows)
    return;
  R *base = reinterpret_cast<R *>(kron_smem) + int64_t(warp) * WS;
  R *bufr[2] = {base, base + 2 * TS};
  R *bufi[2] = {base + TS, base + 3 * TS};
  R *tabs    = base + 4 * TS; // [D][kKronTab]
  // with up to four entries per lane, v's loads are issued first so they
  // overlap the dependent table loads (cell -> table index -> table)
  double vpre[KEEP ? PER : 1];
  if constexpr (KEEP)
  {
#pragma unroll
    for (int o = 0; o < PER; o++)
    {
      int const i = lane + 32 * o;
      vpre[o]     = (i < TS) ? v[int64_t(c) * TS + i] : 0.0;
    }
  }
  for (int e = lane; e < D * kKronTab; e += 32)
  {
    int const k = e / kKronTab;
    tabs[e]     = tab[(int64_t(kself[int64_t(c) * D + k]) * D + k) * kKronTab +
                  (e - k * kKronTab)];
  }
  double const f = scale_state ? scale_state[1] : 1.0;
  unsigned dig[PD]; // base-3 digits, two bits per dimension, dim 0 highest
  auto digit = [&](int o, int i, int k) -> int {
    if constexpr (KEEP)
      return int((dig[o] >> (2 * k)) & 3u);
    else
      return (i / ipow3j(D - 1 - k)) % 3;
  };
#pragma unroll
  for (int o = 0; o < PD; o++)
  {
    int t       = lane + 32 * o;
    unsigned pk = 0;
#pragma unroll
    for (int k = D - 1; k >= 0; k--)
    {
      pk |= unsigned(t % 3) << (2 * k);
      t /= 3;
    }
    dig[o] = pk;
  }
#pragma unroll(KEEP ? PER : 1)
  for (int o = 0; o < PER; o++)
  {
    int const i = lane + 32 * o;
    if (i < TS)
    {
      double vv;
      if constexpr (KEEP)
        vv = vpre[o];
      else
        vv = v[int64_t(c) * TS + i];
      if (scale_state)
      {
        vv                     = vv * f;
        v[int64_t(c) * TS + i] = vv;
        if (vcopy)
          vcopy[int64_t(c) * TS + i] = float(vv);
      }
      bufr[0][i] = R(vv);
      bufi[0][i] = R(0);
    }
  }
  __syncwarp();
  int cur = 0;
  // out = (I (x) M (x) I) in along dimension k, M column-major complex: lane
  // f takes fibre f along k (the three entries that differ only in their
  // k-th index), so every input is read once and M sits in registers
  auto stage = [&](int k, int st, int moff) {
    constexpr int NF = TS / 3;
    const R *mp      = tabs + k * kKronTab + moff;
    R mr[9], mi[9];
#pragma unroll
    for (int e = 0; e < 9; e++)
    {
      mr[e] = mp[2 * e];
      mi[e] = mp[2 * e + 1];
    }
    const R *ir = bufr[cur], *ii = bufi[cur];
    R *orr = bufr[cur ^ 1], *oi = bufi[cur ^ 1];
#pragma unroll(NF <= 32 ? 1 : 2)
    for (int fb = lane; fb < NF; fb += 32)
    {
      int const b0 = (fb / st) * 3 * st + (fb % st);
      R xr[3], xi[3];
#pragma unroll
      for (int pp = 0; pp < 3; pp++)
      {
        xr[pp] = ir[b0 + pp * st];
        xi[pp] = ii[b0 + pp * st];
      }
#pragma unroll
      for (int q = 0; q < 3; q++)
      {
        R yr = R(0), yi = R(0);
#pragma unroll
        for (int pp = 0; pp < 3; pp++)
        {
          yr += mr[q + 3 * pp] * xr[pp] - mi[q + 3 * pp] * xi[pp];
          yi += mr[q + 3 * pp] * xi[pp] + mi[q + 3 * pp] * xr[pp];
        }
        orr[b0 + q * st] = yr;
        oi[b0 + q * st]  = yi;
      }
    }
    cur ^= 1;
    __syncwarp();
  };
#pragma unroll
  for (int k = 0; k < D; k++)
    stage(k, ipow3j(D - 1 - k), 18); // W_k
  {
    R const sh = R(shift), mdt = R(-dt);
    R *ur = bufr[cur], *ui = bufi[cur];
#pragma unroll(KEEP ? PER : 1)
    for (int o = 0; o < PER; o++)
    {
      int const i = lane + 32 * o;
      if (i < TS)
      {
        R mr = sh, mi = R(0);
#pragma unroll
        for (int k = 0; k < D; k++)
        {
          int const q = digit(o, i, k);
          mr += mdt * tabs[k * kKronTab + 36 + 2 * q];
          mi += mdt * tabs[k * kKronTab + 37 + 2 * q];
        }
        R const den = mr * mr + mi * mi;
        R const xr = ur[i], xi = ui[i];
        ur[i] = (xr * mr + xi * mi) / den;
        ui[i] = (xi * mr - xr * mi) / den;
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int k = 0; k < D; k++)
    stage(k, ipow3j(D - 1 - k), 0); // V_k
  for (int o = 0; o < PER; o++)
  {
    int const i = lane + 32 * o;
    if (i < TS)
      z[int64_t(c) * TS + i] = double(bufr[cur][i]);
  }
}

template<typename R, int D>
int launch_kron_apply(int rows, const int *kself, const R *tab, double shift,
                      double dt, double *v, double *z, const double *sc,
                      float *vc, cudaStream_t s)
{
  constexpr int TS  = ipow3j(D);
  constexpr int WPC = TS <= 81 ? 4 : 2;
  size_t const shm  = size_t(WPC) * (4 * TS + D * kKronTab) * sizeof(R);
  auto kern         = k_kron_apply<R, D, WPC>;
  if (shm > 48 * 1024)
    ASGK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(shm)));
  kern<<<(rows + WPC - 1) / WPC, WPC * 32, shm, s>>>(rows, kself, tab, shift, dt,
                                                   v, z, sc, vc, g_gate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

template<typename R>
int kron_apply_r(int d, int rows, const int *kself, const R *tab, double shift,
                 double dt, double *v, double *z, const double *sc,
                 float *vc, cudaStream_t s)
{
  switch (d)
  {
  case 1: return launch_kron_apply<R, 1>(rows, kself, tab, shift, dt, v, z, sc, vc, s);
  case 2: return launch_kron_apply<R, 2>(rows, kself, tab, shift, dt, v, z, sc, vc, s);
  case 3: return launch_kron_apply<R, 3>(rows, kself, tab, shift, dt, v, z, sc, vc, s);
  case 4: return launch_kron_apply<R, 4>(rows, kself, tab, shift, dt, v, z, sc, vc, s);
  case 5: return launch_kron_apply<R, 5>(rows, kself, tab, shift, dt, v, z, sc, vc, s);
  case 6: return launch_kron_apply<R, 6>(rows, kself, tab, shift, dt, v, z, sc, vc, s);
  default: return ASGK_ERR_UNSUPPORTED;
  }
}

using cd = std::complex<double>;

// B V = V diag(lam), W = V^-1, for a real 3x3 b (column-major).  A multiple
// of the identity (a dimension no term acts in) gives V = W = I.  False when
// the eigenvalues are not distinct or a check fails (residual, inverse).
bool eig3(const double *b, cd lam[3], cd V[9], cd W[9])
{
  auto A = [&](int i, int j) { return b[i + 3 * j]; };
  double nb = 0;
  for (int e = 0; e < 9; e++)
    nb = std::max(nb, std::fabs(b[e]));
  bool const scalar = A(1, 0) == 0 && A(2, 0) == 0 && A(0, 1) == 0 &&
                      A(2, 1) == 0 && A(0, 2) == 0 && A(1, 2) == 0 &&
                      A(0, 0) == A(1, 1) && A(1, 1) == A(2, 2);
  if (scalar)
  {
    for (int e = 0; e < 9; e++)
      V[e] = W[e] = cd((e % 4 == 0) ? 1.0 : 0.0);
    lam[0] = lam[1] = lam[2] = cd(A(0, 0));
    return true;
  }
  // characteristic polynomial x^3 + c2 x^2 + c1 x + c0
  double const tr = A(0, 0) + A(1, 1) + A(2, 2);
  double const m  = A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0) + A(0, 0) * A(2, 2) -
                   A(0, 2) * A(2, 0) + A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1);
  double const det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) -
                     A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                     A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
  double const c2 = -tr, c1 = m, c0 = -det;
  auto poly = [&](cd x) { return ((x + c2) * x + c1) * x + c0; };
  auto dpoly = [&](cd x) { return (3.0 * x + 2.0 * c2) * x + c1; };
  // a real root by bisection on the Cauchy bound, then the quadratic
  double lo = -(1 + std::max({std::fabs(c2), std::fabs(c1), std::fabs(c0)}));
  double hi = -lo;
  for (int it = 0; it < 200; it++)
  {
    double const mid = 0.5 * (lo + hi);
    if (poly(cd(mid)).real() > 0)
      hi = mid;
    else
      lo = mid;
  }
  double const r  = 0.5 * (lo + hi);
  double const q1 = c2 + r, q0 = c1 + r * q1;
  cd const sq     = std::sqrt(cd(q1 * q1 - 4 * q0));
  lam[0]          = cd(r);
  lam[1]          = (-q1 + sq) * 0.5;
  lam[2]          = (-q1 - sq) * 0.5;
  for (int e = 0; e < 3; e++) // polish on the cubic
    for (int it = 0; it < 3; it++)
    {
      cd const dp = dpoly(lam[e]);
      if (std::abs(dp) > 0)
        lam[e] -= poly(lam[e]) / dp;
    }
  double const tiny = 1e-300;
  for (int e = 0; e < 3; e++)
    for (int f = e + 1; f < 3; f++)
      if (std::abs(lam[e] - lam[f]) <= 1e-8 * (nb + tiny))
        return false;
  // eigenvectors: the largest cross product of two rows of (A - lam I)
  for (int e = 0; e < 3; e++)
  {
    cd M[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        M[i][j] = cd(A(i, j)) - ((i == j) ? lam[e] : cd(0));
    auto cross = [&](int a, int c, cd out[3]) {
      out[0] = M[a][1] * M[c][2] - M[a][2] * M[c][1];
      out[1] = M[a][2] * M[c][0] - M[a][0] * M[c][2];
      out[2] = M[a][0] * M[c][1] - M[a][1] * M[c][0];
    };
    cd best[3], cur[3];
    double bn = -1;
    int const pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (auto const &pq : pr)
    {
      cross(pq[0], pq[1], cur);
      double const nn = std::abs(cur[0]) + std::abs(cur[1]) + std::abs(cur[2]);
      if (nn > bn)
      {
        bn = nn;
        std::copy(cur, cur + 3, best);
      }
    }
    double const scale = std::sqrt(std::norm(best[0]) + std::norm(best[1]) + std::norm(best[2]));
    if (!(scale > 1e-12 * (nb * nb + tiny)))
      return false;
    for (int i = 0; i < 3; i++)
      V[i + 3 * e] = best[i] / scale;
  }
  // W = V^-1 by the adjugate
  auto v = [&](int i, int j) { return V[i + 3 * j]; };
  cd const dv = v(0, 0) * (v(1, 1) * v(2, 2) - v(1, 2) * v(2, 1)) -
                v(0, 1) * (v(1, 0) * v(2, 2) - v(1, 2) * v(2, 0)) +
                v(0, 2) * (v(1, 0) * v(2, 1) - v(1, 1) * v(2, 0));
  if (!(std::abs(dv) > 1e-6)) // unit columns: |det| is a conditioning measure
    return false;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
    {
      int const i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      // (V^-1)(j, i) = cofactor(i, j) / det
      W[j + 3 * i] = (v(i1, j1) * v(i2, j2) - v(i1, j2) * v(i2, j1)) / dv;
    }
  // checks: A V = V diag(lam) and W V = I
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
    {
      cd av = 0, wv = 0;
      for (int q = 0; q < 3; q++)
      {
        av += A(i, q) * v(q, j);
        wv += W[i + 3 * q] * v(q, j);
      }
      if (std::abs(av - v(i, j) * lam[j]) > 1e-10 * (nb + tiny) ||
          std::abs(wv - cd(i == j ? 1.0 : 0.0)) > 1e-10)
        return false;
    }
  return true;
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
  // kron: per (1D cell, dimension) tables, each cell's self connections
  int d            = 0;
  double kshift    = 0;       // 1 - dt * (number of identity terms)
  double *kt64     = nullptr; // [nconn * d][kKronTab]
  float *kt32      = nullptr;
  int *kself       = nullptr; // [rows * d]
  // line: pencil tables and intermediates (jacobi_line.cu)
  line_data *line  = nullptr;
  int64_t device_bytes = 0;
  ~jacobi_data()
  {
    line_free(line);
    cudaFree(inv_diag);
    cudaFree(M64);
    cudaFree(M16);
    cudaFree(kt64);
    cudaFree(kt32);
    cudaFree(kself);
  }
};

int jacobi_build(plan_data const &p, double dt, int kind, jacobi_data &jd)
{
  if (p.rows != p.cols)
    return ASGK_ERR_INVALID;
  if (kind != ASGK_JACOBI_POINT && kind != ASGK_JACOBI_BLOCK &&
      kind != ASGK_JACOBI_KRON && kind != ASGK_JACOBI_LINE)
    return ASGK_ERR_INVALID;
  int const ts = p.tensor;
  if (kind == ASGK_JACOBI_BLOCK && ts > 81)
    return ASGK_ERR_UNSUPPORTED; // the shared-memory inverse holds ts x 2ts
  // the Kronecker-sum form needs the global form's per-dimension blocks and
  // no term acting in several dimensions
  if (kind == ASGK_JACOBI_KRON && (!p.global || p.gchains > 0 || p.n != 3))
    return ASGK_ERR_UNSUPPORTED;
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
  if (kind == ASGK_JACOBI_LINE)
  {
    jd.d = p.d;
    return line_build(p, dt, &jd.line, jd.device_bytes);
  }
  // the plan's FP64 factors in the layout its indices address
  const double *vA = p.vA64;
  if (kind == ASGK_JACOBI_KRON)
  {
    // eigendecompositions of every self block (one per 1D cell and
    // dimension), from the plan's pre-summed per-dimension blocks
    int const d         = p.d;
    int64_t const nconn = int64_t(p.g_conn_row.size());
    std::vector<double> B(size_t(nconn) * d * 10);
    ASGK_CUDA(cudaMemcpy(B.data(), p.gB64, sizeof(double) * B.size(),
                         cudaMemcpyDeviceToHost));
    std::vector<double> t64(size_t(nconn) * d * kKronTab, 0.0);
    for (int64_t j = 0; j < nconn; j++)
    {
      if (p.g_conn_row[j] != p.g_conn_col[j])
        continue;
      for (int k = 0; k < d; k++)
      {
        cd lam[3], V[9], W[9];
        if (!eig3(&B[size_t(j * d + k) * 10], lam, V, W))
          return ASGK_ERR_UNSUPPORTED;
        double *t = &t64[size_t(j * d + k) * kKronTab];
        for (int e = 0; e < 9; e++)
        {
          t[2 * e]          = V[e].real();
          t[2 * e + 1]      = V[e].imag();
          t[18 + 2 * e]     = W[e].real();
          t[18 + 2 * e + 1] = W[e].imag();
        }
        for (int e = 0; e < 3; e++)
        {
          t[36 + 2 * e]     = lam[e].real();
          t[36 + 2 * e + 1] = lam[e].imag();
        }
      }
    }
    std::vector<float> t32(t64.begin(), t64.end());
    jd.d      = d;
    jd.kshift = 1.0 - dt * p.g_identity;
    ASGK_CUDA(cudaMalloc(&jd.kt64, sizeof(double) * t64.size()));
    ASGK_CUDA(cudaMalloc(&jd.kt32, sizeof(float) * t32.size()));
    ASGK_CUDA(cudaMalloc(&jd.kself, sizeof(int) * size_t(p.rows) * d));
    ASGK_CUDA(cudaMemcpy(jd.kt64, t64.data(), sizeof(double) * t64.size(),
                         cudaMemcpyHostToDevice));
    ASGK_CUDA(cudaMemcpy(jd.kt32, t32.data(), sizeof(float) * t32.size(),
                         cudaMemcpyHostToDevice));
    // the global plan's pair list holds each cell's own pair, with its self
    // connection in every dimension
    ASGK_CUDA(cudaMemcpy(jd.kself, p.idx, sizeof(int) * size_t(p.rows) * d,
                         cudaMemcpyDeviceToDevice));
    jd.device_bytes = int64_t(t64.size() * 12 + size_t(p.rows) * d * 4);
    return ASGK_OK;
  }
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
                 const double *scale_state, float *vcopy, cudaStream_t s,
                 float *zcopy)
{
  int64_t const n = int64_t(jd.rows) * jd.ts;
  if (jd.kind == ASGK_JACOBI_LINE)
    return line_apply(*jd.line, low, v, z, scale_state, vcopy, zcopy, s);
  if (jd.kind == ASGK_JACOBI_KRON)
  {
    if (low)
      return kron_apply_r<float>(jd.d, jd.rows, jd.kself, jd.kt32, jd.kshift,
                                 jd.dt, v, z, scale_state, vcopy, s);
    return kron_apply_r<double>(jd.d, jd.rows, jd.kself, jd.kt64, jd.kshift,
                                jd.dt, v, z, scale_state, vcopy, s);
  }
  if (jd.kind == ASGK_JACOBI_POINT)
  {
    int const blocks = int(std::min<int64_t>((n + 255) / 256, 4096));
    k_point_apply<<<blocks, 256, 0, s>>>(n, jd.inv_diag, v, z, scale_state, vcopy,
                                         g_gate);
    ASGK_LAUNCHED();
    return ASGK_OK;
  }
  if (low)
  {
    if (jd.ps16 / 8 > kApply16Threads * kApply16Loads)
      return ASGK_ERR_UNSUPPORTED;
    size_t const shm = sizeof(__half) * jd.ps16 + sizeof(float) * jd.ts;
    k_block_apply16<<<jd.rows, kApply16Threads, shm, s>>>(jd.ts, jd.ps16, jd.M16, v, z,
                                                          scale_state, vcopy, g_gate);
  }
  else
  {
    int const threads = jd.ts <= 32 ? 32 : (jd.ts <= 64 ? 64 : 128);
    size_t const shm  = sizeof(double) * jd.ts;
    k_block_apply<double><<<jd.rows, threads, shm, s>>>(jd.rows, jd.ts, jd.M64, v, z,
                                                        scale_state, vcopy, g_gate);
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
                              nullptr, static_cast<cudaStream_t>(stream));
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

int asgk_jacobi_apply_precision(asgk_jacobi *pc, int precision,
                                const double *v, double *z, asgk_stream stream)
{
  try
  {
    if (pc == nullptr || v == nullptr || z == nullptr ||
        (precision != ASGK_FP64 && precision != ASGK_FP32))
      return ASGK_ERR_INVALID;
    return asgk::jacobi_apply(pc->jd, precision == ASGK_FP32,
                              const_cast<double *>(v), z, nullptr, nullptr,
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

int asgk::jacobi_check_shape(const asgk_jacobi *pc, int rows, int tensor)
{
  if (pc == nullptr || pc->jd.rows != rows || pc->jd.ts != tensor)
    return ASGK_ERR_INVALID;
  return ASGK_OK;
}

double asgk::jacobi_dt(const asgk_jacobi *pc) { return pc ? pc->jd.dt : 0.0; }

int asgk::jacobi_apply_handle(asgk_jacobi *pc, bool low, double *v, double *z,
                              const double *scale_state, float *vcopy,
                              cudaStream_t s, float *zcopy)
{
  return asgk::jacobi_apply(pc->jd, low, v, z, scale_state, vcopy, s, zcopy);
}

bool asgk::jacobi_writes_zcopy(const asgk_jacobi *pc)
{
  return pc != nullptr && pc->jd.kind == ASGK_JACOBI_LINE;
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
