// Global-mode kronmult apply (n = 3): the operator applied through the cell
// pairs that differ in at most one dimension -- terms acting in one
// dimension in one pass, terms acting in several as chains of masked 1D
// passes (the reference's upper/lower permutations).
//
// Reference: the global Kronecker form (global_kron_matrix,
// src/asgard_kronmult_matrix.cpp:1196-1334; global_cpu_one,
// src/device/asgard_glkronmult_cpu.cpp:103-181).  For a term whose factors
// are the identity in all dimensions but k, the term's product over the
// connected-pair list equals one 1D operator along k: a pair contributes
// only when its cells agree in every dimension other than k (an identity
// block between different 1D cells is zero).  The reference applies such a
// term as one sparse product along k over all degrees of freedom (its
// "both" fill, no upper/lower split); here a CTA owns an output cell (cells
// with the most neighbours first), its warps walk the cell's neighbours along
// single dimensions and apply each pre-summed 3x3 block to the neighbour's
// tensor along that dimension:
//   y_r = beta y_r + alpha * (sum_{(c, k)} (I (x) B_k[conn] (x) I) x_c
//                             + n_identity x_r) + ex x_r.
// 2 * 3^(d+1) flops per entry; the neighbour tensors come from L2.
#include "internal.cuh"

#include <algorithm>
#include <cstdint>

namespace asgk
{
namespace
{
constexpr int ipow3g(int k) { return k == 0 ? 1 : 3 * ipow3g(k - 1); }


template<typename TC> struct padG;
template<> struct padG<double> { static constexpr int value = 10; };
template<> struct padG<float> { static constexpr int value = 12; };

// Stride of dimension k in a 3^D tensor (dimension 0 slowest), 3^(D-1-k):
// byte k of the packed constant.
template<int D>
__device__ __forceinline__ int dim_stride(int k)
{
  constexpr unsigned long long packed =
      D == 1 ? 0x01ull : D == 2 ? 0x0103ull : D == 3 ? 0x010309ull
      : D == 4 ? 0x0103091bull : D == 5 ? 0x0103091b51ull : 0x0103091b51f3ull;
  return int((packed >> (8 * k)) & 0xff);
}

// One CTA per slice of at most kSlice (64) entries of an output cell's
// neighbour list.  A cell's entries come in
// dimension order; for the entries along dimension k, lane f of a warp owns
// fibre f of the 3^d tensor along k (the three entries that differ only in
// their k-th index): it loads the neighbour's fibre and applies the 3x3 block
// to it, accumulating in registers, and adds its three sums into the warp's
// row of shared memory when the dimension changes.  The NW warps take the
// slice's entries in turn (four in flight per warp); their rows are summed
// at the end.  A cell with one slice writes y at once; the slices of a cell
// with several write partial tensors to scratch, and the last of them to
// finish (an atomic ticket, no waiting) adds them in slice order and writes
// y -- deterministic whichever slice ends last.
template<int D, typename TC, int NW, int kSlice>
__global__ void __launch_bounds__(NW * 32)
    kron_global_rows(const int *__restrict__ slice_row,
                     const int64_t *__restrict__ slice_beg,
                     const int *__restrict__ slice_len,
                     const int *__restrict__ row_slice0,
                     const int *__restrict__ row_nslice,
                     const int *__restrict__ gcol, const int *__restrict__ gkb,
                     const TC *__restrict__ B, double *__restrict__ scratch,
                     unsigned *__restrict__ tickets, double alpha,
                     const double *__restrict__ x, double beta,
                     double *__restrict__ y, double ex,
                     const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  constexpr int TS  = ipow3g(D);
  constexpr int NF  = TS / 3;           // fibres along one dimension
  constexpr int FPL = (NF + 31) / 32;   // fibres per lane
  constexpr int PAD = padG<TC>::value;
  constexpr int NT  = NW * 32;
  __shared__ TC red[NW * TS];
  __shared__ int s_col[kSlice], s_kb[kSlice];
  __shared__ int s_seg[D + 1];
  __shared__ unsigned s_ticket;

  int const warp   = threadIdx.x >> 5;
  int const lane   = threadIdx.x & 31;
  int const sl     = blockIdx.x;
  int const row    = slice_row[sl];
  int const s0     = row_slice0[row];
  int const ns     = row_nslice[row];
  int64_t const eb = slice_beg[sl];
  int const n      = slice_len[sl];

  // the slice's entries come in dimension order: s_seg[k] is the first
  // entry along dimension k or after (s_seg[D] = n), written by the entry
  // that opens the segment
  for (int i = threadIdx.x; i < n; i += NT)
  {
    int const kb = __ldg(gkb + eb + i);
    s_col[i]     = __ldg(gcol + eb + i);
    s_kb[i]      = kb;
    int const dk = kb % D;
    int const dp = (i > 0) ? __ldg(gkb + eb + i - 1) % D : -1;
    for (int k = dp + 1; k <= dk; k++)
      s_seg[k] = i;
    if (i == n - 1)
      for (int k = dk + 1; k <= D; k++)
        s_seg[k] = n;
  }
  if (n == 0 && threadIdx.x <= D)
    s_seg[threadIdx.x] = 0;
  for (int i = threadIdx.x; i < NW * TS; i += NT)
    red[i] = TC(0);
  __syncthreads();

  TC *myred = red + warp * TS;
  for (int k = 0; k < D; k++)
  {
    int const sa = s_seg[k], sb = s_seg[k + 1];
    if (sa == sb)
      continue;
    int const stride = dim_stride<D>(k);
    int fb[FPL]; // first entry of each fibre this lane owns
    TC acc[FPL][3];
#pragma unroll
    for (int m = 0; m < FPL; m++)
    {
      int const f = lane + 32 * m;
      fb[m]       = (f / stride) * 3 * stride + (f % stride);
      acc[m][0] = acc[m][1] = acc[m][2] = TC(0);
    }
    auto entry = [&](int j) {
      const TC *b      = B + int64_t(s_kb[j]) * PAD;
      const double *xc = x + int64_t(s_col[j]) * TS;
      // the padded block (12 floats / 10 doubles) in 16-byte loads
      TC b0, b1, b2, b3, b4, b5, b6, b7, b8;
      if constexpr (sizeof(TC) == 4)
      {
        const float4 *q = reinterpret_cast<const float4 *>(b);
        float4 const q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
        b0 = q0.x, b1 = q0.y, b2 = q0.z, b3 = q0.w;
        b4 = q1.x, b5 = q1.y, b6 = q1.z, b7 = q1.w;
        b8 = q2.x;
      }
      else
      {
        const double2 *q = reinterpret_cast<const double2 *>(b);
        double2 const q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
        double2 const q3 = __ldg(q + 3), q4 = __ldg(q + 4);
        b0 = q0.x, b1 = q0.y, b2 = q1.x, b3 = q1.y, b4 = q2.x;
        b5 = q2.y, b6 = q3.x, b7 = q3.y, b8 = q4.x;
      }
#pragma unroll
      for (int m = 0; m < FPL; m++)
      {
        if (lane + 32 * m < NF)
        {
          TC const v0 = static_cast<TC>(__ldg(xc + fb[m]));
          TC const v1 = static_cast<TC>(__ldg(xc + fb[m] + stride));
          TC const v2 = static_cast<TC>(__ldg(xc + fb[m] + 2 * stride));
          // column-major block: out_q += sum_p A(q, p) v_p, A(q, p) = b[q + 3p]
          acc[m][0] = fma(b6, v2, fma(b3, v1, fma(b0, v0, acc[m][0])));
          acc[m][1] = fma(b7, v2, fma(b4, v1, fma(b1, v0, acc[m][1])));
          acc[m][2] = fma(b8, v2, fma(b5, v1, fma(b2, v0, acc[m][2])));
        }
      }
    };
    for (int j = sa + warp; j < sb; j += 4 * NW)
    {
      entry(j);
      if (j + NW < sb)
        entry(j + NW);
      if (j + 2 * NW < sb)
        entry(j + 2 * NW);
      if (j + 3 * NW < sb)
        entry(j + 3 * NW);
    }
    // lanes own distinct fibres: their outputs along k do not overlap
#pragma unroll
    for (int m = 0; m < FPL; m++)
      if (lane + 32 * m < NF)
      {
        myred[fb[m]] += acc[m][0];
        myred[fb[m] + stride] += acc[m][1];
        myred[fb[m] + 2 * stride] += acc[m][2];
      }
    __syncwarp(); // before the next dimension's fibres touch these entries
  }
  __syncthreads();
  int64_t const base = int64_t(row) * TS;
  if (ns == 1)
  {
    for (int i = threadIdx.x; i < TS; i += NT)
    {
      TC s = TC(0);
#pragma unroll
      for (int w = 0; w < NW; w++)
        s += red[w * TS + i];
      double v = alpha * static_cast<double>(s) + ex * x[base + i];
      if (beta != 0.0)
        v += beta * y[base + i];
      y[base + i] = v;
    }
    return;
  }
  // several slices: publish this slice's partial tensor
  double *mine = scratch + int64_t(sl) * TS;
  for (int i = threadIdx.x; i < TS; i += NT)
  {
    TC s = TC(0);
#pragma unroll
    for (int w = 0; w < NW; w++)
      s += red[w * TS + i];
    mine[i] = static_cast<double>(s);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0)
    s_ticket = atomicAdd(tickets + row, 1u);
  __syncthreads();
  if (s_ticket != unsigned(ns - 1))
    return;
  // the last slice of the row: add the slices in order, finish the row
  __threadfence();
  for (int i = threadIdx.x; i < TS; i += NT)
  {
    double s = 0.0;
    for (int q = 0; q < ns; q++)
      s += __ldcg(scratch + int64_t(s0 + q) * TS + i);
    double v = alpha * s + ex * x[base + i];
    if (beta != 0.0)
      v += beta * y[base + i];
    y[base + i] = v;
  }
  if (threadIdx.x == 0)
    tickets[row] = 0u; // ready for the next launch
}

// d >= 5, FP32: one CTA per output cell, warp k takes the cell's neighbours
// along dimension k (no barrier until the end): lane f owns fibres f,
// f + 32, ... of the 3^d tensor along k, loads each neighbour's fibre (from
// the FP32 copy of x in the FP32 apply: 47 MB at d=6, level 7, held in L2
// across the re-reads) and accumulates the 3x3 block's product in
// registers; the warps' results meet in shared memory and are added in
// dimension order with the Euler term (from the staged copy of the cell's
// own tensor, 94 MB of FP64 reads fewer per apply at d=6, level 7) and the
// beta term (FP64 y).  The lane's
// fibres are taken in PASSES passes over the warp's entries: with two, half
// the accumulators are live, so six CTAs fit on an SM instead of four
// (measured at d=6, level 7: 0.344 -> 0.317 ms with the conversion pass;
// three or four passes spill and are slower).  The cell's own tensor is
// staged in shared memory once, for the self entry of every dimension
// (0.317 -> 0.304 ms).
template<int D, typename TC, typename TX, int PASSES>
__global__ void __launch_bounds__(D * 32, PASSES == 1 ? 4 : 6)
    kron_global_cell_dims(const int *__restrict__ order,
                     const int64_t *__restrict__ gptr,
                     const int *__restrict__ gseg, const int *__restrict__ gcol,
                     const int *__restrict__ gkb, const TC *__restrict__ B,
                     double alpha, const TX *__restrict__ xs,
                     const double *__restrict__ x, double beta,
                     double *__restrict__ y, double ex,
                     const double *__restrict__ gate)
{
  (void)x; // the Euler term reads the staged copy
  if (gate_closed(gate))
    return;
  constexpr int TS  = ipow3g(D);
  constexpr int NF  = TS / 3;
  constexpr int FPL = (NF + 31) / 32;
  constexpr int PAD = padG<TC>::value;
  __shared__ TC rows[D * TS];
  __shared__ TX own[TS]; // the cell's own tensor: every warp's self entry
  int const k    = threadIdx.x >> 5;
  int const lane = threadIdx.x & 31;
  int const cell = order[blockIdx.x];
  for (int i = threadIdx.x; i < TS; i += D * 32)
    own[i] = xs[int64_t(cell) * TS + i];
  __syncthreads();
  int64_t const e0 = gptr[cell];
  int const sa = gseg[cell * (D + 1) + k], sb = gseg[cell * (D + 1) + k + 1];
  int const stride = dim_stride<D>(k);
  // the lane's fibres f = lane + 32 m, m < FPL, in PASSES passes over the
  // warp's entries (fewer live registers per pass, more warps per SM)
  constexpr int FPP = (FPL + PASSES - 1) / PASSES;
  TC *row = rows + k * TS;
#pragma unroll 1
  for (int pass = 0; pass < PASSES; pass++)
  {
  int fb[FPP];
  TC acc[FPP][3];
#pragma unroll
  for (int m = 0; m < FPP; m++)
  {
    int const f = lane + 32 * (pass * FPP + m);
    fb[m]       = (f / stride) * 3 * stride + (f % stride);
    acc[m][0] = acc[m][1] = acc[m][2] = TC(0);
  }
  auto live = [&](int m) { return pass * FPP + m < FPL && lane + 32 * (pass * FPP + m) < NF; };
  auto entry = [&](int64_t j) {
    const TC *b  = B + int64_t(__ldg(gkb + j)) * PAD;
    int const c  = __ldg(gcol + j);
    const TX *xc = xs + int64_t(c) * TS;
    TC b0, b1, b2, b3, b4, b5, b6, b7, b8;
    if constexpr (sizeof(TC) == 4)
    {
      const float4 *q = reinterpret_cast<const float4 *>(b);
      float4 const q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
      b0 = q0.x, b1 = q0.y, b2 = q0.z, b3 = q0.w;
      b4 = q1.x, b5 = q1.y, b6 = q1.z, b7 = q1.w;
      b8 = q2.x;
    }
    else
    {
      const double2 *q = reinterpret_cast<const double2 *>(b);
      double2 const q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
      double2 const q3 = __ldg(q + 3), q4 = __ldg(q + 4);
      b0 = q0.x, b1 = q0.y, b2 = q1.x, b3 = q1.y, b4 = q2.x;
      b5 = q2.y, b6 = q3.x, b7 = q3.y, b8 = q4.x;
    }
    TC v[FPP][3];
    if (c == cell) // warp-uniform: the self entry reads the staged tensor
    {
#pragma unroll
      for (int m = 0; m < FPP; m++)
        if (live(m))
#pragma unroll
          for (int p = 0; p < 3; p++)
            v[m][p] = static_cast<TC>(own[fb[m] + p * stride]);
    }
    else
    {
#pragma unroll
      for (int m = 0; m < FPP; m++)
        if (live(m))
#pragma unroll
          for (int p = 0; p < 3; p++)
            v[m][p] = static_cast<TC>(__ldg(xc + fb[m] + p * stride));
    }
#pragma unroll
    for (int m = 0; m < FPP; m++)
      if (live(m))
      {
        // column-major block: out_q += sum_p A(q, p) v_p, A(q, p) = b[q + 3p]
        acc[m][0] = fma(b6, v[m][2], fma(b3, v[m][1], fma(b0, v[m][0], acc[m][0])));
        acc[m][1] = fma(b7, v[m][2], fma(b4, v[m][1], fma(b1, v[m][0], acc[m][1])));
        acc[m][2] = fma(b8, v[m][2], fma(b5, v[m][1], fma(b2, v[m][0], acc[m][2])));
      }
  };
  for (int j = sa; j < sb; j++)
    entry(e0 + j);
#pragma unroll
  for (int m = 0; m < FPP; m++)
    if (live(m))
    {
      row[fb[m]]              = acc[m][0];
      row[fb[m] + stride]     = acc[m][1];
      row[fb[m] + 2 * stride] = acc[m][2];
    }
  }
  __syncthreads();
  int64_t const base = int64_t(cell) * TS;
  for (int i = threadIdx.x; i < TS; i += D * 32)
  {
    TC s = TC(0);
#pragma unroll
    for (int kk = 0; kk < D; kk++)
      s += rows[kk * TS + i];
    // the Euler term from the staged tensor: the operand of the whole
    // low-precision apply (x rounded as the neighbour tensors are), and no
    // second read of the FP64 x
    double v = alpha * static_cast<double>(s) + ex * static_cast<double>(own[i]);
    if (beta != 0.0)
      v += beta * y[base + i];
    y[base + i] = v;
  }
}

// d >= 5, FP64: one CTA per output cell, D warps sharing the cell's
// neighbour list (in dimension order) in equal contiguous ranges, so no
// warp waits on another's long dimension (measured at d=6, level 7: 0.64 ->
// 0.46 ms; the FP32 apply, which reads from L2, is faster with a warp per
// dimension).  Within a dimension k lane f owns fibres f,
// f + 32, ... of the 3^d tensor along k, loads each neighbour's fibre (from
// the FP32 copy of x in the FP32 apply: 47 MB at d=6, level 7, held in L2
// across the re-reads) and accumulates the 3x3 block's product in
// registers; when its range moves on to the next dimension the warp adds
// its sums into its own row of shared memory.  The rows are added in warp
// order with the Euler and beta terms (FP64 x and y): a fixed order, the
// same result whichever warp finishes first.  A lane's fibres are taken in
// PASSES passes over each segment (two: 80 registers, four CTAs per SM,
// 0.439 -> 0.422 ms at d=6, level 7).
template<int D, typename TC, typename TX, int PASSES>
__global__ void __launch_bounds__(D * 32, PASSES == 1 ? 2 : 4)
    kron_global_cell_ranges(const int *__restrict__ order,
                     const int64_t *__restrict__ gptr,
                     const int *__restrict__ gseg, const int *__restrict__ gcol,
                     const int *__restrict__ gkb, const TC *__restrict__ B,
                     double alpha, const TX *__restrict__ xs,
                     const double *__restrict__ x, double beta,
                     double *__restrict__ y, double ex,
                     const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  constexpr int TS  = ipow3g(D);
  constexpr int NF  = TS / 3;
  constexpr int FPL = (NF + 31) / 32;
  constexpr int PAD = padG<TC>::value;
  __shared__ TC rows[D * TS];
  int const w    = threadIdx.x >> 5;
  int const lane = threadIdx.x & 31;
  int const cell = order[blockIdx.x];
  int64_t const e0 = gptr[cell];
  int const E  = gseg[cell * (D + 1) + D];
  int const ja = int(int64_t(E) * w / D), jb = int(int64_t(E) * (w + 1) / D);
  int k = 0; // the dimension of the range's first entry
  while (k < D - 1 && gseg[cell * (D + 1) + k + 1] <= ja)
    ++k;
  TC *row = rows + w * TS;
  for (int i = lane; i < TS; i += 32)
    row[i] = TC(0);
  __syncwarp();
  int j = ja;
  while (j < jb)
  {
    int const send   = min(jb, gseg[cell * (D + 1) + k + 1]);
    int const stride = dim_stride<D>(k);
    // the lane's fibres in PASSES passes over the segment's entries
    constexpr int FPP = (FPL + PASSES - 1) / PASSES;
    int const jseg = j;
#pragma unroll 1
    for (int pass = 0; pass < PASSES; pass++)
    {
    auto live = [&](int m) { return pass * FPP + m < FPL && lane + 32 * (pass * FPP + m) < NF; };
    int fb[FPP];
    TC acc[FPP][3];
#pragma unroll
    for (int m = 0; m < FPP; m++)
    {
      int const f = lane + 32 * (pass * FPP + m);
      fb[m]       = (f / stride) * 3 * stride + (f % stride);
      acc[m][0] = acc[m][1] = acc[m][2] = TC(0);
    }
    for (j = jseg; j < send; j++)
    {
      int64_t const e = e0 + j;
      const TC *b  = B + int64_t(__ldg(gkb + e)) * PAD;
      const TX *xc = xs + int64_t(__ldg(gcol + e)) * TS;
      TC b0, b1, b2, b3, b4, b5, b6, b7, b8;
      if constexpr (sizeof(TC) == 4)
      {
        const float4 *q = reinterpret_cast<const float4 *>(b);
        float4 const q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
        b0 = q0.x, b1 = q0.y, b2 = q0.z, b3 = q0.w;
        b4 = q1.x, b5 = q1.y, b6 = q1.z, b7 = q1.w;
        b8 = q2.x;
      }
      else
      {
        const double2 *q = reinterpret_cast<const double2 *>(b);
        double2 const q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
        double2 const q3 = __ldg(q + 3), q4 = __ldg(q + 4);
        b0 = q0.x, b1 = q0.y, b2 = q1.x, b3 = q1.y, b4 = q2.x;
        b5 = q2.y, b6 = q3.x, b7 = q3.y, b8 = q4.x;
      }
      TC v[FPP][3];
#pragma unroll
      for (int m = 0; m < FPP; m++)
        if (live(m))
#pragma unroll
          for (int p = 0; p < 3; p++)
            v[m][p] = static_cast<TC>(__ldg(xc + fb[m] + p * stride));
#pragma unroll
      for (int m = 0; m < FPP; m++)
        if (live(m))
        {
          // column-major block: out_q += sum_p A(q, p) v_p, A(q, p) = b[q + 3p]
          acc[m][0] = fma(b6, v[m][2], fma(b3, v[m][1], fma(b0, v[m][0], acc[m][0])));
          acc[m][1] = fma(b7, v[m][2], fma(b4, v[m][1], fma(b1, v[m][0], acc[m][1])));
          acc[m][2] = fma(b8, v[m][2], fma(b5, v[m][1], fma(b2, v[m][0], acc[m][2])));
        }
    }
    // lanes own distinct fibres of dimension k: no two lanes touch an entry
#pragma unroll
    for (int m = 0; m < FPP; m++)
      if (live(m))
      {
        row[fb[m]] += acc[m][0];
        row[fb[m] + stride] += acc[m][1];
        row[fb[m] + 2 * stride] += acc[m][2];
      }
    }
    __syncwarp(); // before the next dimension's fibres touch these entries
    ++k;
  }
  __syncthreads();
  int64_t const base = int64_t(cell) * TS;
  for (int i = threadIdx.x; i < TS; i += D * 32)
  {
    TC s = TC(0);
#pragma unroll
    for (int ww = 0; ww < D; ww++)
      s += rows[ww * TS + i];
    double v = alpha * static_cast<double>(s) + ex * x[base + i];
    if (beta != 0.0)
      v += beta * y[base + i];
    y[base + i] = v;
  }
}

// the FP32 copy of x the FP32 cell kernel reads; pairs of values when x is
// 16-byte aligned, single values otherwise (a basis column of an odd-length
// system)
__global__ void k_copy_to_f32(int64_t n, const double *__restrict__ x,
                              float *__restrict__ x32, int pairs,
                              const double *__restrict__ gate)
{
  if (gate_closed(gate))
    return;
  int64_t const t0 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  int64_t const ts = int64_t(gridDim.x) * blockDim.x;
  if (pairs)
  {
    for (int64_t i = t0; i < n / 2; i += ts)
    {
      double2 const v = reinterpret_cast<const double2 *>(x)[i];
      reinterpret_cast<float2 *>(x32)[i] = make_float2(float(v.x), float(v.y));
    }
    if (t0 == 0 && (n & 1))
      x32[n - 1] = float(x[n - 1]);
  }
  else
    for (int64_t i = t0; i < n; i += ts)
      x32[i] = float(x[i]);
}

// One stage of the chains of the terms acting in several dimensions
// (src/device/asgard_glkronmult_cpu.cpp:103-181): for job (chain, dimension
// k, fill, term) and output cell r,
//   out_r = sum over r's neighbours c along k of block(r, c), masked by the
//           fill, applied along k to in_c,
// where block(r, c) is the term's 3x3 factor of dimension k for the 1D pair
// (r_k, c_k).  The fill splits the 1D operator at its diagonal, in the
// order (1D cell, polynomial) of the reference's sparsity pattern: upper
// keeps the neighbours after r_k and, on r_k itself, the columns p >= q of
// row q; lower keeps the neighbours before r_k and the columns p < q.
// in_stride 0: every job reads the same input (stage 0 reads x).
template<int D, typename TC, typename TX>
__global__ void __launch_bounds__(128)
    kron_global_chain(const int4 *__restrict__ jobs, int rows,
                      const int64_t *__restrict__ dptr,
                      const int *__restrict__ dcol,
                      const int *__restrict__ dconn,
                      const unsigned char *__restrict__ drel,
                      const TC *__restrict__ P, int T,
                      const TX *__restrict__ in, int64_t in_stride,
                      TC *__restrict__ out, int64_t N)
{
  constexpr int TS  = ipow3g(D);
  constexpr int PAD = padG<TC>::value;
  int4 const job    = jobs[blockIdx.y];
  int const chain   = job.x, k = job.y, fill = job.z, t = job.w;
  int const r       = blockIdx.x;
  const TX *src     = in + int64_t(chain) * in_stride;
  TC *o             = out + int64_t(chain) * N + int64_t(r) * TS;
  int64_t const b0  = dptr[int64_t(k) * (rows + 1) + r];
  int64_t const b1  = dptr[int64_t(k) * (rows + 1) + r + 1];
  int const stride  = dim_stride<D>(k);
  for (int i = threadIdx.x; i < TS; i += blockDim.x)
  {
    int const q    = (i / stride) % 3;
    int const base = i - q * stride;
    TC acc         = TC(0);
    for (int64_t e = b0; e < b1; e++)
    {
      int const rel = drel[e];
      int plo = 0, phi = 3;
      if (fill == 0) // upper
      {
        if (rel == 0)
          continue;
        if (rel == 1)
          plo = q;
      }
      else if (fill == 2) // lower
      {
        if (rel == 2)
          continue;
        if (rel == 1)
          phi = q;
      }
      const TC *b  = P + ((int64_t(dconn[e]) * D + k) * T + t) * PAD;
      const TX *xc = src + int64_t(dcol[e]) * TS + base;
      for (int pp = plo; pp < phi; pp++)
        acc = fma(__ldg(b + q + 3 * pp), static_cast<TC>(xc[pp * stride]), acc);
    }
    o[i] = acc;
  }
}

// y += alpha * (sum of the chains' results), chains in order
template<typename TC>
__global__ void k_chain_sum(int chains, const int *__restrict__ last,
                            const TC *__restrict__ work, int64_t N,
                            double alpha, double *__restrict__ y)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < N;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    double s = 0.0;
    for (int c = 0; c < chains; c++)
      s += static_cast<double>(work[(int64_t(last[c]) * chains + c) * N + i]);
    y[i] += alpha * s;
  }
}

template<int D, typename TC>
int launch_chains(plan_data const &p, double alpha, const double *x, double *y,
                  cudaStream_t s)
{
  constexpr int TS  = ipow3g(D);
  int const threads = TS >= 128 ? 128 : (TS + 31) / 32 * 32;
  const TC *P;
  if constexpr (sizeof(TC) == 8)
    P = p.vP64;
  else
    P = p.vP32;
  int64_t const N = int64_t(p.rows) * TS;
  TC *work        = reinterpret_cast<TC *>(p.gwork);
  for (size_t st = 0; st < p.stage_njobs.size(); st++)
  {
    dim3 const grid(p.rows, p.stage_njobs[st]);
    const int4 *jobs = p.gjobs + p.stage_job0[st];
    TC *out          = work + int64_t(st % 2) * p.gchains * N;
    if (st == 0)
      kron_global_chain<D, TC, double><<<grid, threads, 0, s>>>(
          jobs, p.rows, p.gd_ptr, p.gd_col, p.gd_conn, p.gd_rel, P, p.terms, x,
          0, out, N);
    else
      kron_global_chain<D, TC, TC><<<grid, threads, 0, s>>>(
          jobs, p.rows, p.gd_ptr, p.gd_col, p.gd_conn, p.gd_rel, P, p.terms,
          work + int64_t((st - 1) % 2) * p.gchains * N, N, out, N);
    ASGK_LAUNCHED();
  }
  int const blocks = int(std::min<int64_t>((N + 255) / 256, 4096));
  k_chain_sum<TC><<<blocks, 256, 0, s>>>(p.gchains, p.gchain_last, work, N, alpha, y);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

template<int D, typename TC>
int launch_global_d(plan_data const &p, double alpha, const double *x,
                    double beta, double *y, double ex, cudaStream_t s)
{
  constexpr int TS    = ipow3g(D);
  constexpr int NW    = TS <= 81 ? 4 : 8;
  constexpr int SLICE = global_slice(D);
  static_assert(SLICE <= kGlobalSliceMax, "slice");
  const TC *B;
  if constexpr (sizeof(TC) == 8)
    B = p.gB64;
  else
    B = p.gB32;
  if constexpr (D >= 5)
  {
    if (p.gseg != nullptr)
    {
      int64_t const n = int64_t(p.rows) * TS;
      if constexpr (sizeof(TC) == 4)
      {
        // the copy is already there when the preconditioner wrote it with x
        if (p.gx32_src != x)
        {
          int const pairs  = (reinterpret_cast<uintptr_t>(x) % 16) == 0 ? 1 : 0;
          int const blocks = int(std::min<int64_t>((n / 2 + 255) / 256, 4 * 148));
          k_copy_to_f32<<<blocks, 256, 0, s>>>(n, x, p.gx32, pairs, g_gate);
          ASGK_LAUNCHED();
        }
        p.gx32_src = nullptr;
        kron_global_cell_dims<D, TC, float, 2><<<p.rows, D * 32, 0, s>>>(
            p.gcell_order, p.gptr, p.gseg, p.gcol, p.gkb, B, alpha, p.gx32, x, beta, y,
            ex, g_gate);
      }
      else
        kron_global_cell_ranges<D, TC, double, 2><<<p.rows, D * 32, 0, s>>>(
            p.gcell_order + p.rows, p.gptr, p.gseg, p.gcol, p.gkb, B, alpha, x, x, beta,
            y, ex, g_gate);
      ASGK_LAUNCHED();
      if (p.gchains > 0)
        return launch_chains<D, TC>(p, alpha, x, y, s);
      return ASGK_OK;
    }
  }
  kron_global_rows<D, TC, NW, SLICE><<<p.gslices, NW * 32, 0, s>>>(
      p.slice_row, p.slice_beg, p.slice_len, p.row_slice0, p.row_nslice, p.gcol, p.gkb, B,
      p.gscratch, p.gtickets, alpha, x, beta, y, ex, g_gate);
  ASGK_LAUNCHED();
  if (p.gchains > 0)
    return launch_chains<D, TC>(p, alpha, x, y, s);
  return ASGK_OK;
}

template<typename TC>
int launch_global_t(plan_data const &p, double alpha, const double *x,
                    double beta, double *y, double ex, cudaStream_t s)
{
  switch (p.d)
  {
  case 1: return launch_global_d<1, TC>(p, alpha, x, beta, y, ex, s);
  case 2: return launch_global_d<2, TC>(p, alpha, x, beta, y, ex, s);
  case 3: return launch_global_d<3, TC>(p, alpha, x, beta, y, ex, s);
  case 4: return launch_global_d<4, TC>(p, alpha, x, beta, y, ex, s);
  case 5: return launch_global_d<5, TC>(p, alpha, x, beta, y, ex, s);
  case 6: return launch_global_d<6, TC>(p, alpha, x, beta, y, ex, s);
  default: return ASGK_ERR_UNSUPPORTED;
  }
}

} // namespace

int launch_global(plan_data const &p, int precision, double alpha,
                  const double *x, double beta, double *y, double ex,
                  cudaStream_t s)
{
  if (p.n != 3 || (g_gate != nullptr && p.gchains > 0))
    return ASGK_ERR_UNSUPPORTED; // the chain kernels take no gate
  // terms that are the identity in every dimension add n_identity * x
  double const ex_eff = ex + alpha * p.g_identity;
  int rc = ASGK_ERR_UNSUPPORTED;
  if (precision == ASGK_FP64)
    rc = launch_global_t<double>(p, alpha, x, beta, y, ex_eff, s);
  else if (precision == ASGK_FP32)
    rc = launch_global_t<float>(p, alpha, x, beta, y, ex_eff, s);
  else if (precision == ASGK_BF16)
  {
    rc = tc_prepare(p);
    if (rc == ASGK_OK)
      rc = launch_global_tc(p, alpha, x, beta, y, ex_eff, s);
  }
  p.gx32_src = nullptr; // a preconditioner's copy serves the next apply only
  return rc;
}

} // namespace asgk
