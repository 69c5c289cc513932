// Line preconditioner (ASGK_JACOBI_LINE) of the backward-Euler operator
// I - dt*K for global plans whose terms act in one dimension each.  No
// counterpart in the reference, whose only preconditioner is the diagonal
// one (src/solver.cpp:76-91).
//
// K = sum_k K_k, K_k the terms acting in dimension k.  K_k couples only
// cells that agree outside dimension k (a "pencil" along k), and on a
// pencil it is A_k restricted to the pencil's 1D cells (x) I on the other
// dimensions.  On a standard sparse grid a pencil holds every 1D cell of
// level <= L' along k, so its matrix is a leading principal submatrix of the
// 1D operator A_k: one per pencil level.  For the "line" dimensions -- those
// whose 1D operator is symmetric (the stiff diffusion terms) -- the solve
//   M_k = s I - dt (K_k + sum_{j line, j != k} D_j),  D_j: cell-diagonal part of K_j,
// s = 1 - dt * (identity terms), is exact per pencil: with A_P = Q diag(theta)
// Q^T (A_P the pencil's submatrix) and the 3x3 self blocks of the other line
// dimensions S_j = P_j diag(lambda_j) P_j^T (constant over the pencil: its
// cells share their 1D cells outside k), all orthogonal,
//   M_k^-1 = (Q (x) (x)_j P_j) diag(1 / (s - dt (theta + sum_j lambda_j))) (Q^T (x) (x)_j P_j^T)
// on each group of values with fixed polynomial indices in the non-line
// dimensions.  The preconditioner chains the line dimensions k_1 < ... < k_m:
//   z = M_{k_m}^-1 B ... B M_{k_2}^-1 B M_{k_1}^-1 v,   B = s I - dt sum_{j line} D_j,
// an alternating-direction product whose factors each invert one diffusion
// direction exactly; dimensions with non-symmetric operators (advection)
// are left to GMRES.  Each factor is one kernel launch over (pencil, group
// range) units: gather the unit's values, apply B (factors after the first),
// transform the columns by the P_j^T and the rows by Q^T (a dense product,
// the pencil matrix read through L2), divide, transform back, scatter.  The
// first factor also normalises v and writes its FP32 copy inside recorded
// GMRES cycles; intermediates live in two vectors held by the
// preconditioner; no atomics (each value belongs to exactly one unit).
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <new>
#include <numeric>
#include <type_traits>
#include <vector>

namespace asgk
{
namespace
{
constexpr int kLineItems   = 128;            // item slots of a factor CTA
constexpr int kLineThreads = 2 * kLineItems; // two halves share each item
constexpr int kGatherLoads = 8; // loads in flight per thread while gathering
constexpr int kSelfEntry   = 21; // P (3x3 col-major), lambda (3), S (3x3 col-major)

constexpr int ipow3l(int k) { return k <= 0 ? 1 : 3 * ipow3l(k - 1); }

// Symmetric eigendecomposition by cyclic Jacobi rotations: A (n x n,
// row-major, symmetric) = V diag(w) V^T with V orthogonal (eigenvectors in
// its columns, row-major storage).  Each rotation zeroes one off-diagonal
// entry a_pq: tau = (a_qq - a_pp) / (2 a_pq), t = sign(tau) / (|tau| +
// sqrt(1 + tau^2)), c = 1/sqrt(1 + t^2), s = t c.
bool sym_eig(int n, std::vector<double> A, std::vector<double> &V,
             std::vector<double> &w)
{
  V.assign(size_t(n) * n, 0.0);
  for (int i = 0; i < n; i++)
    V[size_t(i) * n + i] = 1.0;
  double norm = 0;
  for (double a : A)
    norm += a * a;
  norm = std::sqrt(norm);
  for (int sweep = 0; sweep < 60; sweep++)
  {
    double off = 0;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++)
        off += A[size_t(p) * n + q] * A[size_t(p) * n + q];
    if (std::sqrt(2 * off) <= 1e-15 * norm || norm == 0.0)
    {
      w.resize(n);
      for (int i = 0; i < n; i++)
        w[i] = A[size_t(i) * n + i];
      return true;
    }
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++)
      {
        double const apq = A[size_t(p) * n + q];
        if (std::abs(apq) <= 1e-300 ||
            std::abs(apq) <= 1e-18 * (std::abs(A[size_t(p) * n + p]) +
                                      std::abs(A[size_t(q) * n + q])))
          continue;
        double const tau = (A[size_t(q) * n + q] - A[size_t(p) * n + p]) / (2 * apq);
        double const t   = (tau >= 0 ? 1.0 : -1.0) / (std::abs(tau) + std::sqrt(1 + tau * tau));
        double const c   = 1 / std::sqrt(1 + t * t), s = t * c;
        for (int k = 0; k < n; k++)
        {
          double const akp = A[size_t(k) * n + p], akq = A[size_t(k) * n + q];
          A[size_t(k) * n + p] = c * akp - s * akq;
          A[size_t(k) * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++)
        {
          double const apk = A[size_t(p) * n + k], aqk = A[size_t(q) * n + k];
          A[size_t(p) * n + k] = c * apk - s * aqk;
          A[size_t(q) * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++)
        {
          double const vkp = V[size_t(k) * n + p], vkq = V[size_t(k) * n + q];
          V[size_t(k) * n + p] = c * vkp - s * vkq;
          V[size_t(k) * n + q] = s * vkp + c * vkq;
        }
      }
  }
  return false;
}

// Everything a factor launch reads (device pointers; the tables typed by R).
template<typename R>
struct line_args
{
  const int4 *units;  // (pencil, first group, groups, 0)
  const int *pen_off; // into pen_cells
  const int *pen_m;   // members
  const int *pen_tab; // pencil matrix table
  const int *pen_cells;
  const int *c1;      // [cells][D] 1D cell of every cell in every dimension
  const int *tab_off; // into Q / QT (each Rr x Rp)
  const int *tab_th;  // into theta
  const int *tab_rp;
  const R *Q, *QT, *theta;
  const R *self;      // [line index][1D cells][kSelfEntry]
  int r1;             // number of 1D cells
  int k, kidx;        // this factor's dimension and its index among the line dims
  int line[3];        // line dimensions (increasing)
  int nonline[6];     // the other dimensions (increasing)
  int st_k;           // tensor stride of dimension k, 3^(D-1-k)
  int st_line[3];     // tensor strides of the line dimensions
  R shift, dt;
};

template<typename R> struct vec4_of;
template<> struct vec4_of<float>
{
  static __device__ __forceinline__ void load(const float *p, float q[4])
  {
    float4 const v = __ldg(reinterpret_cast<const float4 *>(p));
    q[0] = v.x, q[1] = v.y, q[2] = v.z, q[3] = v.w;
  }
};
template<> struct vec4_of<double>
{
  static __device__ __forceinline__ void load(const double *p, double q[4])
  {
    double2 const a = __ldg(reinterpret_cast<const double2 *>(p));
    double2 const b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    q[0] = a.x, q[1] = a.y, q[2] = b.x, q[3] = b.y;
  }
};

// 16-byte asynchronous global->shared copies (no L1 allocation), in
// groups the waits below count
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
  unsigned const sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit()
{
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template<int N>
__device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kLineTile = 16; // matrix rows per staged tile

// a = fma(qa, x, a), b = fma(qb, x, b): for FP32 one packed two-lane FMA
// (fma.rn.f32x2, each lane rounded as the scalar FMA, so the same bits)
__device__ __forceinline__ void fma_pair(float qa, float qb, float x, float &a, float &b)
{
  asm("{\n\t.reg .b64 rq, rx, ra;\n\t"
      "mov.b64 rq, {%2, %3};\n\tmov.b64 rx, {%4, %4};\n\tmov.b64 ra, {%0, %1};\n\t"
      "fma.rn.f32x2 ra, rq, rx, ra;\n\tmov.b64 {%0, %1}, ra;\n\t}"
      : "+f"(a), "+f"(b)
      : "f"(qa), "f"(qb), "f"(x));
}
__device__ __forceinline__ void fma_pair(double qa, double qb, double x, double &a, double &b)
{
  a = fma(qa, x, a);
  b = fma(qb, x, b);
}

// shared-memory rows read in 16-byte pieces (rows start 16-byte aligned)
__device__ __forceinline__ void smem_row4(const float *p, float (&q)[4])
{
  float4 const v = *reinterpret_cast<const float4 *>(p);
  q[0] = v.x, q[1] = v.y, q[2] = v.z, q[3] = v.w;
}
__device__ __forceinline__ void smem_row4(const double *p, double (&q)[4])
{
  double2 const a = reinterpret_cast<const double2 *>(p)[0];
  double2 const b = reinterpret_cast<const double2 *>(p)[1];
  q[0] = a.x, q[1] = a.y, q[2] = b.x, q[3] = b.y;
}
template<typename R, int N>
__device__ __forceinline__ void smem_row(const R *p, R (&q)[N])
{
  if constexpr (N % 4 == 0)
  {
#pragma unroll
    for (int i = 0; i < N / 4; i++)
    {
      R t[4];
      smem_row4(p + 4 * i, t);
#pragma unroll
      for (int e = 0; e < 4; e++)
        q[4 * i + e] = t[e];
    }
  }
  else
  {
#pragma unroll
    for (int i = 0; i < N; i++)
      q[i] = p[i];
  }
}

// out[r][g][c] = sum_{t < Rr} Mt[t][r] in[t][g][c] for r < Rr (Mt rows of
// Rp entries, zero beyond Rr, in global memory), divided by den(r, c) when
// theta is given.  Mt streams through shared memory in tiles of kLineTile
// rows, double-buffered with cp.async.  The (4-row block, group) items go
// to kLineItems thread slots, at most two each, their sums in registers
// across the tiles; the two halves of the block take the first and second
// half of every tile's rows for the same items, so each thread's chain of
// dependent tiles is half as long.  The second half leaves its partial
// sums in out, where the first adds them to its own (a fixed order) and
// finishes.
template<typename R, int NC, int NCP>
__device__ void dense_rows(const R *__restrict__ Mt, int Rr, int Rp, int G,
                           const R *__restrict__ in, R *__restrict__ out,
                           const R *__restrict__ theta, const R *lamc, R shift,
                           R dt, R *qbuf)
{
  constexpr int TH = kLineTile / 2; // rows of a tile per half
  int const rb_n  = Rp / 4;
  int const items = rb_n * G;
  int const tiles = (Rr + kLineTile - 1) / kLineTile;
  int const chunks_per_row = Rp * int(sizeof(R)) / 16;
  int const half = threadIdx.x / kLineItems, slot = threadIdx.x % kLineItems;
  auto issue = [&](int tile) {
    int const t0 = tile * kLineTile;
    int const nr = min(kLineTile, Rr - t0);
    R *dst       = qbuf + (tile & 1) * kLineTile * Rp;
    const char *src = reinterpret_cast<const char *>(Mt + int64_t(t0) * Rp);
    for (int c = threadIdx.x; c < nr * chunks_per_row; c += blockDim.x)
      cp_async16(reinterpret_cast<char *>(dst) + 16 * c, src + 16 * c);
    cp_async_commit();
  };
  int const it0 = slot, it1 = slot + kLineItems;
  bool const has0 = it0 < items, has1 = it1 < items;
  int const rb0 = has0 ? it0 % rb_n : 0, g0 = has0 ? it0 / rb_n : 0;
  int const rb1 = has1 ? it1 % rb_n : 0, g1 = has1 ? it1 / rb_n : 0;
  R acc0[4][NC], acc1[4][NC];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int c = 0; c < NC; c++)
      acc0[i][c] = acc1[i][c] = R(0);
  issue(0);
  for (int tile = 0; tile < tiles; tile++)
  {
    if (tile + 1 < tiles)
    {
      issue(tile + 1);
      cp_async_wait<1>();
    }
    else
      cp_async_wait<0>();
    __syncthreads();
    int const t0 = tile * kLineTile;
    int const nr = min(kLineTile, Rr - t0);
    const R *qt  = qbuf + (tile & 1) * kLineTile * Rp;
#pragma unroll
    for (int th = 0; th < TH; th++)
    {
      int const tt = half * TH + th;
      if (tt >= nr)
        break;
      int const t = t0 + tt;
      if (has0)
      {
        R q[4], xv[NCP];
        smem_row4(qt + tt * Rp + 4 * rb0, q);
        smem_row<R, NCP>(in + (int64_t(t) * G + g0) * NCP, xv);
#pragma unroll
        for (int c = 0; c < NC; c++)
        {
          fma_pair(q[0], q[1], xv[c], acc0[0][c], acc0[1][c]);
          fma_pair(q[2], q[3], xv[c], acc0[2][c], acc0[3][c]);
        }
      }
      if (has1)
      {
        R q[4], xv[NCP];
        smem_row4(qt + tt * Rp + 4 * rb1, q);
        smem_row<R, NCP>(in + (int64_t(t) * G + g1) * NCP, xv);
#pragma unroll
        for (int c = 0; c < NC; c++)
        {
          fma_pair(q[0], q[1], xv[c], acc1[0][c], acc1[1][c]);
          fma_pair(q[2], q[3], xv[c], acc1[2][c], acc1[3][c]);
        }
      }
    }
    __syncthreads(); // the buffer is refilled two tiles on
  }
  auto at = [&](int r, int g, int c) { return out + (int64_t(r) * G + g) * NCP + c; };
  auto park = [&](int rb, int g, R (&acc)[4][NC]) {
#pragma unroll
    for (int i = 0; i < 4; i++)
    {
      int const r = 4 * rb + i;
      if (r >= Rr)
        break;
#pragma unroll
      for (int c = 0; c < NC; c++)
        *at(r, g, c) = acc[i][c];
    }
  };
  auto finish = [&](int rb, int g, R (&acc)[4][NC]) {
#pragma unroll
    for (int i = 0; i < 4; i++)
    {
      int const r = 4 * rb + i;
      if (r >= Rr)
        break;
      R th = R(0);
      if (theta)
        th = __ldg(theta + r);
#pragma unroll
      for (int c = 0; c < NC; c++)
      {
        R v = acc[i][c] + *at(r, g, c);
        if (theta)
          v = v / (shift - dt * (th + lamc[c]));
        *at(r, g, c) = v;
      }
    }
  };
  if (half == 1)
  {
    if (has0)
      park(rb0, g0, acc0);
    if (has1)
      park(rb1, g1, acc1);
  }
  __syncthreads();
  if (half == 0)
  {
    if (has0)
      finish(rb0, g0, acc0);
    if (has1)
      finish(rb1, g1, acc1);
  }
}

// One factor M_k^-1 (after B when bj) on the (pencil, group range) units.
// D dimensions, M line dimensions; NC = 3^(M-1) columns per group (the other
// line dimensions' polynomials), groups: the 3^(D-M) polynomial indices of
// the non-line dimensions.
template<typename R, int D, int M, int KIDX>
__global__ void __launch_bounds__(kLineThreads)
    k_line_factor(line_args<R> a, const double *in64,
                  const R *__restrict__ inR, double *__restrict__ out64,
                  R *__restrict__ outR, int bj, const double *scale_state,
                  double *vscale, float *vcopy, float *__restrict__ zcopy,
                  const double *gate)
{
  if (gate_closed(gate))
    return;
  constexpr int TS  = ipow3l(D);
  constexpr int NC  = ipow3l(M - 1);
  constexpr int NCP = NC == 1 ? 1 : (NC == 3 ? 4 : 12);
  constexpr int NNL = D - M; // non-line dimensions
  extern __shared__ __align__(16) unsigned char line_smem[];
  int4 const u   = a.units[blockIdx.x];
  int const pen  = u.x, g0 = u.y, G = u.z;
  int const m    = a.pen_m[pen];
  int const tab  = a.pen_tab[pen];
  int const Rr   = 3 * m;
  int const Rp   = a.tab_rp[tab];
  const int *cells = a.pen_cells + a.pen_off[pen];
  // per (member, group): its cell's offset plus the group's digits in the
  // vector, and its first row of X -- so gathering and scattering divide by
  // no run-time size
  int64_t *s_rowoff = reinterpret_cast<int64_t *>(line_smem);
  int *s_xrow       = reinterpret_cast<int *>(s_rowoff + m * G);
  R *X = reinterpret_cast<R *>(line_smem + ((12 * size_t(m) * G + 15) / 16) * 16);
  R *Y    = X + int64_t(Rp) * G * NCP;
  R *qbuf = Y + int64_t(Rp) * G * NCP; // 2 tiles of kLineTile matrix rows
  __shared__ int s_offg[27];
  __shared__ int s_offc[NC];
  __shared__ R s_lamc[NC];
  __shared__ R s_P[3][9]; // other line dimensions' eigenvectors (P_j, col-major)
  __shared__ R s_S[3][9]; // their self blocks (B, all line dimensions)
  int const cell0 = cells[0];
  // offsets of the group and column digits in a cell's tensor (dimension 0
  // slowest); the other line dimensions' eigen data, constant over the pencil
  if (threadIdx.x < G)
  {
    int g = g0 + threadIdx.x, off = 0;
    for (int q = NNL - 1; q >= 0; q--)
    {
      off += (g % 3) * ipow3l(D - 1 - a.nonline[q]);
      g /= 3;
    }
    s_offg[threadIdx.x] = off;
  }
  if (threadIdx.x < NC)
  {
    int c = threadIdx.x, off = 0;
    R lam = R(0);
    for (int q = M - 1; q >= 0; q--)
    {
      if (q == KIDX)
        continue;
      int const j  = a.line[q];
      int const dg = c % 3;
      c /= 3;
      off += dg * ipow3l(D - 1 - j);
      lam += a.self[(int64_t(q) * a.r1 + a.c1[int64_t(cell0) * D + j]) * kSelfEntry + 9 + dg];
    }
    s_offc[threadIdx.x] = off;
    s_lamc[threadIdx.x] = lam;
  }
  if (threadIdx.x < 9 * M)
  {
    int const q = threadIdx.x / 9, e = threadIdx.x % 9;
    int const j = a.line[q];
    const R *sf = a.self + (int64_t(q) * a.r1 + a.c1[int64_t(cell0) * D + j]) * kSelfEntry;
    s_P[q][e] = sf[e];
    s_S[q][e] = sf[12 + e];
  }
  __syncthreads();
  for (int it = threadIdx.x; it < m * G; it += blockDim.x)
  {
    int const i  = it / G, g = it - i * G;
    s_rowoff[it] = int64_t(__ldg(cells + i)) * TS + s_offg[g];
    s_xrow[it]   = (i * 3 * G + g) * NCP;
  }
  __syncthreads();
  int const stk = ipow3l(D - 1 - a.k);
  double const f = scale_state ? scale_state[1] : 1.0;
  // gather (row = member * 3 + k polynomial, group, column); kGatherLoads
  // independent loads per thread are issued before their values are used
  int const nload = m * G * 3 * NC;
  auto gidx = [&](int e, int &xo) {
    int const ig = e / (3 * NC), w = e - ig * (3 * NC);
    int const pk = w / NC, c = w - pk * NC;
    xo           = s_xrow[ig] + pk * G * NCP + c;
    return s_rowoff[ig] + s_offc[c] + pk * stk;
  };
  for (int e0 = threadIdx.x; e0 < nload; e0 += kGatherLoads * kLineThreads)
  {
    int64_t gi[kGatherLoads];
    int xo[kGatherLoads];
#pragma unroll
    for (int u = 0; u < kGatherLoads; u++)
    {
      int const e = e0 + u * kLineThreads;
      gi[u]       = e < nload ? gidx(e, xo[u]) : 0;
    }
    if (in64)
    {
      double v[kGatherLoads];
#pragma unroll
      for (int u = 0; u < kGatherLoads; u++)
        if (e0 + u * kLineThreads < nload)
          v[u] = in64[gi[u]];
#pragma unroll
      for (int u = 0; u < kGatherLoads; u++)
      {
        if (e0 + u * kLineThreads >= nload)
          break;
        double vv = v[u];
        if (scale_state)
        {
          vv *= f;
          vscale[gi[u]] = vv;
          if (vcopy)
            vcopy[gi[u]] = float(vv);
        }
        X[xo[u]] = R(vv);
      }
    }
    else
    {
      R v[kGatherLoads];
#pragma unroll
      for (int u = 0; u < kGatherLoads; u++)
        if (e0 + u * kLineThreads < nload)
          v[u] = inR[gi[u]];
#pragma unroll
      for (int u = 0; u < kGatherLoads; u++)
        if (e0 + u * kLineThreads < nload)
          X[xo[u]] = v[u];
    }
  }
  __syncthreads();
  // B = s - dt sum_{line j} S_j along j, on each (member, group): its 3 x NC
  // values are the cell's line-dimension polynomials
  if (bj)
  {
    for (int it = threadIdx.x; it < m * G; it += blockDim.x)
    {
      int const i = it / G, g = it % G;
      R v[3][NC], o[3][NC];
#pragma unroll
      for (int pk = 0; pk < 3; pk++)
#pragma unroll
        for (int c = 0; c < NC; c++)
          v[pk][c] = X[((int64_t(i) * 3 + pk) * G + g) * NCP + c];
      // this member's own self block along k
      R Sk[9];
      const R *sf = a.self + (int64_t(KIDX) * a.r1 +
                              a.c1[int64_t(cells[i]) * D + a.k]) * kSelfEntry + 12;
#pragma unroll
      for (int e = 0; e < 9; e++)
        Sk[e] = sf[e];
#pragma unroll
      for (int pk = 0; pk < 3; pk++)
#pragma unroll
        for (int c = 0; c < NC; c++)
        {
          R acc = a.shift * v[pk][c];
          // along k: sum_p S_k(pk, p) v[p][c]
          acc -= a.dt * (Sk[pk] * v[0][c] + Sk[pk + 3] * v[1][c] + Sk[pk + 6] * v[2][c]);
          // along the other line dimensions: the column digits
          int stride = 1;
#pragma unroll
          for (int q = M - 1; q >= 0; q--)
          {
            if (q == KIDX)
              continue;
            int const dg = (c / stride) % 3;
            int const cb = c - dg * stride;
            R s = R(0);
#pragma unroll
            for (int p = 0; p < 3; p++)
              s += s_S[q][dg + 3 * p] * v[pk][cb + p * stride];
            acc -= a.dt * s;
            stride *= 3;
          }
          o[pk][c] = acc;
        }
#pragma unroll
      for (int pk = 0; pk < 3; pk++)
#pragma unroll
        for (int c = 0; c < NC; c++)
          X[((int64_t(i) * 3 + pk) * G + g) * NCP + c] = o[pk][c];
    }
    __syncthreads();
  }
  // columns: u <- P_j^T u along every other line dimension, per (row, group)
  auto columns = [&](R *buf, bool forward) {
    if constexpr (NC > 1)
    {
      for (int it = threadIdx.x; it < Rr * G; it += blockDim.x)
      {
        R *row = buf + int64_t(it) * NCP;
        R v[NC];
#pragma unroll
        for (int c = 0; c < NC; c++)
          v[c] = row[c];
        int stride = 1;
#pragma unroll
        for (int q = M - 1; q >= 0; q--)
        {
          if (q == KIDX)
            continue;
          R w[NC];
#pragma unroll
          for (int c = 0; c < NC; c++)
          {
            int const dg = (c / stride) % 3;
            int const cb = c - dg * stride;
            R s = R(0);
#pragma unroll
            for (int p = 0; p < 3; p++)
              // forward: (P^T u)_dg = sum_p P(p, dg) u_p; back: (P u)_dg = sum_p P(dg, p) u_p
              s += (forward ? s_P[q][p + 3 * dg] : s_P[q][dg + 3 * p]) * v[cb + p * stride];
            w[c] = s;
          }
#pragma unroll
          for (int c = 0; c < NC; c++)
            v[c] = w[c];
          stride *= 3;
        }
#pragma unroll
        for (int c = 0; c < NC; c++)
          row[c] = v[c];
      }
      __syncthreads();
    }
  };
  columns(X, true);
  int64_t const to = a.tab_off[tab];
  // rows: Y = Q^T X, divided; then X = Q Y
  dense_rows<R, NC, NCP>(a.Q + to, Rr, Rp, G, X, Y, a.theta + a.tab_th[tab], s_lamc,
                         a.shift, a.dt, qbuf);
  __syncthreads();
  dense_rows<R, NC, NCP>(a.QT + to, Rr, Rp, G, Y, X, nullptr, s_lamc, a.shift,
                         a.dt, qbuf);
  __syncthreads();
  columns(X, false);
  // scatter
  for (int e = threadIdx.x; e < nload; e += blockDim.x)
  {
    int xo;
    int64_t const gi = gidx(e, xo);
    R const val      = X[xo];
    if (out64)
    {
      out64[gi] = double(val);
      if (zcopy)
        zcopy[gi] = float(val);
    }
    else
      outR[gi] = val;
  }
}

// Pencils of at most kSmallMaxM cells: a CTA stages whole cells (up to
// kSmallCells, from pencils of one size) in shared memory with coalesced
// loads and, per pencil column -- one fibre along k in every cell of the
// pencil -- runs the pencil solve in registers.  With W the other line
// dimensions' eigenvector transform, M_k^-1 B = W (Q D^-1 Q^T) Bt W^T where
// Bt = mu I - dt S_k along k (mu = s - dt sum_{j line, j != k} lambda_j of the
// column's polynomial indices, S_k the cell's own self block along k): W^T
// as fibre stages over the staged cells, then Bt, Q^T, the division by
// mu - dt theta and Q in registers per column, then W.
constexpr int kSmallThreads = 128;
constexpr int kSmallCells   = 8;
constexpr int kSmallMaxM    = 8;
constexpr int kSmallMaxR    = 3 * kSmallMaxM;
constexpr int kStageLoads   = 8; // loads in flight per thread while staging

// four consecutive entries of a shared-memory row (16-byte aligned).  The
// loads are volatile so that the compiler reloads the matrix for every
// column instead of hoisting all of it out of the column loop into
// registers (which spills)
__device__ __forceinline__ void lds4(const float *p, float (&q)[4])
{
  unsigned const a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n"
               : "=f"(q[0]), "=f"(q[1]), "=f"(q[2]), "=f"(q[3])
               : "r"(a));
}
__device__ __forceinline__ void lds4(const double *p, double (&q)[4])
{
  unsigned const a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n"
               : "=d"(q[0]), "=d"(q[1])
               : "r"(a));
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n"
               : "=d"(q[2]), "=d"(q[3])
               : "r"(a + 16u));
}

template<typename R, int D, int M, int KIDX, int MC>
__device__ __forceinline__ void small_column(line_args<R> const &a, R *buf,
                                             int slot0, int fb, unsigned dig,
                                             int stk, const R *Qm, const R *inv,
                                             bool bj, const R (*s_Sk)[9],
                                             const R (*s_lam)[2][3])
{
  constexpr int TS = ipow3l(D);
  constexpr int RR = 3 * MC;
  constexpr int RP = (RR + 3) / 4 * 4;
  R x[RR];
#pragma unroll
  for (int i = 0; i < MC; i++)
#pragma unroll
    for (int pk = 0; pk < 3; pk++)
      x[3 * i + pk] = buf[(slot0 + i) * TS + fb + pk * stk];
  // mu from the other line dimensions' polynomial indices of this column
  R mu = a.shift;
#pragma unroll
  for (int qq = 0; qq < M - 1; qq++)
    mu -= a.dt * s_lam[slot0][qq][(dig >> (2 * qq)) & 3u];
  if (bj)
  {
#pragma unroll
    for (int i = 0; i < MC; i++)
    {
      R const x0 = x[3 * i], x1 = x[3 * i + 1], x2 = x[3 * i + 2];
      const R *S = s_Sk[slot0 + i];
#pragma unroll
      for (int pk = 0; pk < 3; pk++)
        x[3 * i + pk] = mu * x[3 * i + pk] - a.dt * (S[pk] * x0 + S[pk + 3] * x1 + S[pk + 6] * x2);
    }
  }
  // Qm: the pencil matrix's eigenvectors staged in shared memory, [t][r]
  // with rows of RP entries.  u = Q^T x row by row of Qm (four entries per
  // load), u_r /= mu - dt theta_r, then out_t = Qm[t, :] u; every sum runs
  // over increasing t (resp. r)
  R u[RP];
#pragma unroll
  for (int r = 0; r < RP; r++)
    u[r] = R(0);
#pragma unroll
  for (int t = 0; t < RR; t++)
#pragma unroll
    for (int r4 = 0; r4 < RP / 4; r4++)
    {
      R q[4];
      lds4(Qm + t * RP + 4 * r4, q);
      fma_pair(q[0], q[1], x[t], u[4 * r4], u[4 * r4 + 1]);
      fma_pair(q[2], q[3], x[t], u[4 * r4 + 2], u[4 * r4 + 3]);
    }
  // 1 / (mu - dt theta_r) from the batch's table: this pencil, this
  // column's digits in the other line dimensions
  unsigned const combo = (M == 3) ? (dig & 3u) + 3u * ((dig >> 2) & 3u) : (M == 2 ? (dig & 3u) : 0u);
  const R *iv = inv + combo * (3 * kSmallCells) + (slot0 / MC) * RR;
#pragma unroll
  for (int r = 0; r < RR; r++)
    u[r] = u[r] * iv[r];
  // two outputs (rows t, t + 1 of Qm) per pass
#pragma unroll
  for (int t = 0; t < RR; t += 2)
  {
    R o0 = R(0), o1 = R(0);
#pragma unroll
    for (int r4 = 0; r4 < RP / 4; r4++)
    {
      R qa[4], qb[4];
      lds4(Qm + t * RP + 4 * r4, qa);
      if (t + 1 < RR)
        lds4(Qm + (t + 1) * RP + 4 * r4, qb);
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (4 * r4 + i < RR)
        {
          if (t + 1 < RR)
            fma_pair(qa[i], qb[i], u[4 * r4 + i], o0, o1);
          else
            o0 = fma(qa[i], u[4 * r4 + i], o0);
        }
    }
    buf[(slot0 + t / 3) * TS + fb + (t % 3) * stk] = o0;
    if (t + 1 < RR)
      buf[(slot0 + (t + 1) / 3) * TS + fb + ((t + 1) % 3) * stk] = o1;
  }
}

// One launch per factor for every batch of small pencils.  A batch record
// holds (pencils, cells per pencil, matrix offset, eigenvalue offset); its
// cells' records (cell, offsets of the cell's self-block entries in the
// line dimensions) follow in batch order, so the staging needs no chain of
// dependent lookups.
template<typename R, int D, int M, int KIDX>
__global__ void __launch_bounds__(kSmallThreads, 6)
    k_line_small(line_args<R> a, const int4 *__restrict__ batches,
                 const int4 *__restrict__ bcells, const double *in64,
                 const R *__restrict__ inR, double *__restrict__ out64,
                 R *__restrict__ outR, int bj, const double *scale_state,
                 double *vscale, float *vcopy, float *__restrict__ zcopy,
                 const double *gate)
{
  if (gate_closed(gate))
    return;
  constexpr int TS = ipow3l(D);
  constexpr int NF = TS / 3;
  extern __shared__ __align__(16) unsigned char line_small_smem[];
  R *buf = reinterpret_cast<R *>(line_small_smem);
  __shared__ int s_cell[kSmallCells];
  // per fibre index: the first entry of the fibre along k and along each
  // other line dimension, and the column's polynomial digits in the other
  // line dimensions (packed two bits each) -- computed once, so the loops
  // below do no integer division by run-time strides
  __shared__ short s_fbk[NF];
  __shared__ short s_fbo[2][NF];
  __shared__ unsigned char s_dig[NF];
  __shared__ __align__(16) R s_Q[kSmallMaxR * kSmallMaxR];
  __shared__ R s_th[kSmallMaxR];
  __shared__ R s_P[kSmallCells][2][9];
  __shared__ R s_lam[kSmallCells][2][3];
  __shared__ R s_Sk[kSmallCells][9];
  // 1 / (mu - dt theta_r) per digit combination of the other line
  // dimensions, pencil and eigenmode (pencils x modes = 3 x cells <= 24)
  __shared__ R s_inv[9 * 3 * kSmallCells];
  // with three line dimensions: the first entries of the 3 x 3 blocks the
  // two other line dimensions span (one item of the merged column stage)
  constexpr int NB9 = TS / 9 > 0 ? TS / 9 : 1;
  __shared__ short s_b9[NB9];
  int4 const bt  = batches[blockIdx.x];
  int const npen = bt.x, MC = bt.y;
  int const nc   = npen * MC;
  int const RR   = 3 * MC, Rp = (RR + 3) / 4 * 4;
  int const tid  = threadIdx.x;
  int const stk  = a.st_k;
  if (tid < nc)
  {
    int4 const cr = bcells[blockIdx.x * kSmallCells + tid];
    s_cell[tid]   = cr.x;
    int const so[3] = {cr.y, cr.z, cr.w};
    // the other line dimensions' eigenvectors and eigenvalues (constant over
    // a pencil) and the cell's own self block along k
    for (int qq = 0; qq < M - 1; qq++)
    {
      const R *sf = a.self + so[qq < KIDX ? qq : qq + 1];
      for (int e = 0; e < 9; e++)
        s_P[tid][qq][e] = sf[e];
      for (int e = 0; e < 3; e++)
        s_lam[tid][qq][e] = sf[9 + e];
    }
    const R *sk = a.self + so[KIDX] + 12;
    for (int e = 0; e < 9; e++)
      s_Sk[tid][e] = sk[e];
  }
  // the batch's pencil matrix (every pencil of a batch has the same one)
  for (int e = tid; e < RR * Rp; e += blockDim.x)
    s_Q[e] = a.Q[bt.z + e];
  if (tid < RR)
    s_th[tid] = a.theta[bt.w + tid];
  for (int fi = tid; fi < NF; fi += blockDim.x)
  {
    int const fb = (fi / stk) * 3 * stk + fi % stk;
    s_fbk[fi]    = short(fb);
    unsigned dg  = 0;
    for (int qq = 0; qq < M - 1; qq++)
    {
      int const sj  = a.st_line[qq < KIDX ? qq : qq + 1];
      s_fbo[qq][fi] = short((fi / sj) * 3 * sj + fi % sj);
      dg |= unsigned((fb / sj) % 3) << (2 * qq);
    }
    s_dig[fi] = (unsigned char)dg;
  }
  int const o0 = 0 < KIDX ? 0 : 1, o1 = 1 < KIDX ? 1 : 2; // the other line dims
  if constexpr (M == 3)
  {
    for (int u = tid; u < NB9; u += blockDim.x)
    {
      int rem = u, idx = 0;
      for (int dim = D - 1; dim >= 0; dim--)
      {
        if (dim == a.line[o0] || dim == a.line[o1])
          continue;
        idx += (rem % 3) * ipow3l(D - 1 - dim);
        rem /= 3;
      }
      s_b9[u] = short(idx);
    }
  }
  __syncthreads();
  {
    constexpr int NCMB = M == 3 ? 9 : (M == 2 ? 3 : 1);
    int const per = npen * RR;
    for (int e = tid; e < NCMB * per; e += blockDim.x)
    {
      int const combo = e / per, rem = e - combo * per;
      int const pi = rem / RR, r = rem - pi * RR;
      int const slot0 = pi * MC;
      unsigned const dig = (M == 3) ? unsigned(combo % 3) | (unsigned(combo / 3) << 2)
                                    : unsigned(combo);
      R mu = a.shift;
      for (int qq = 0; qq < M - 1; qq++)
        mu -= a.dt * s_lam[slot0][qq][(dig >> (2 * qq)) & 3u];
      s_inv[combo * (3 * kSmallCells) + rem] = R(1) / (mu - a.dt * s_th[r]);
    }
  }
  // stage the cells, a warp per cell: kStageLoads independent loads per
  // thread are issued before their values are used, so enough of them are
  // in flight
  constexpr int PER = (TS + 31) / 32;
  int const warp = tid >> 5, lane = tid & 31;
  for (int c = warp; c < nc; c += kSmallThreads / 32)
  {
    int64_t const gb = int64_t(s_cell[c]) * TS;
    R *bc            = buf + c * TS;
    for (int j0 = 0; j0 < PER; j0 += kStageLoads)
    {
      if (in64)
      {
        double v[kStageLoads];
#pragma unroll
        for (int u = 0; u < kStageLoads; u++)
        {
          int const i = lane + 32 * (j0 + u);
          if (j0 + u < PER && i < TS)
            v[u] = in64[gb + i];
        }
        double const f = scale_state ? scale_state[1] : 1.0;
#pragma unroll
        for (int u = 0; u < kStageLoads; u++)
        {
          int const i = lane + 32 * (j0 + u);
          if (j0 + u < PER && i < TS)
          {
            double vv = v[u];
            if (scale_state)
            {
              vv *= f;
              vscale[gb + i] = vv;
              if (vcopy)
                vcopy[gb + i] = float(vv);
            }
            bc[i] = R(vv);
          }
        }
      }
      else
      {
        R v[kStageLoads];
#pragma unroll
        for (int u = 0; u < kStageLoads; u++)
        {
          int const i = lane + 32 * (j0 + u);
          if (j0 + u < PER && i < TS)
            v[u] = inR[gb + i];
        }
#pragma unroll
        for (int u = 0; u < kStageLoads; u++)
        {
          int const i = lane + 32 * (j0 + u);
          if (j0 + u < PER && i < TS)
            bc[i] = v[u];
        }
      }
    }
  }
  __syncthreads();
  // W^T (forward) or W (backward): fibre stages along the other line dimensions
  auto other_stages = [&](bool forward) {
    if constexpr (M == 3)
    {
      // both other line dimensions in one pass over 3 x 3 blocks: along the
      // first (qq = 0), then the second, the same sums as two passes
      int const s1 = a.st_line[o0], s2 = a.st_line[o1];
      for (int it = tid; it < nc * NB9; it += blockDim.x)
      {
        int const slot = it / NB9, u = it - slot * NB9;
        int const base = slot * TS + s_b9[u];
        R v[3][3];
#pragma unroll
        for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
          for (int d2 = 0; d2 < 3; d2++)
            v[d1][d2] = buf[base + d1 * s1 + d2 * s2];
        const R *P = s_P[slot][0];
        R w[3][3];
#pragma unroll
        for (int d2 = 0; d2 < 3; d2++)
#pragma unroll
          for (int o = 0; o < 3; o++)
            w[o][d2] = forward ? P[3 * o] * v[0][d2] + P[3 * o + 1] * v[1][d2] + P[3 * o + 2] * v[2][d2]
                               : P[o] * v[0][d2] + P[o + 3] * v[1][d2] + P[o + 6] * v[2][d2];
        P = s_P[slot][1];
#pragma unroll
        for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
          for (int o = 0; o < 3; o++)
            buf[base + d1 * s1 + o * s2] =
                forward ? P[3 * o] * w[d1][0] + P[3 * o + 1] * w[d1][1] + P[3 * o + 2] * w[d1][2]
                        : P[o] * w[d1][0] + P[o + 3] * w[d1][1] + P[o + 6] * w[d1][2];
      }
      __syncthreads();
    }
    else
    {
    for (int qq = 0; qq < M - 1; qq++)
    {
      int const sj = a.st_line[qq < KIDX ? qq : qq + 1];
      for (int it = tid; it < nc * NF; it += blockDim.x)
      {
        int const slot = it / NF, fi = it - slot * NF;
        int const base = slot * TS + s_fbo[qq][fi];
        R const x0 = buf[base], x1 = buf[base + sj], x2 = buf[base + 2 * sj];
        const R *P = s_P[slot][qq];
#pragma unroll
        for (int o = 0; o < 3; o++)
          buf[base + o * sj] = forward ? P[3 * o] * x0 + P[3 * o + 1] * x1 + P[3 * o + 2] * x2
                                       : P[o] * x0 + P[o + 3] * x1 + P[o + 6] * x2;
      }
      __syncthreads();
    }
    }
  };
  other_stages(true);
  // the pencil solves, one column (fibre along k) per item
  for (int it = tid; it < npen * NF; it += blockDim.x)
  {
    int const pi = it / NF, fi = it - pi * NF;
    switch (MC)
    {
    case 1: small_column<R, D, M, KIDX, 1>(a, buf, pi, s_fbk[fi], s_dig[fi], stk, s_Q, s_inv, bj, s_Sk, s_lam); break;
    case 2: small_column<R, D, M, KIDX, 2>(a, buf, pi * 2, s_fbk[fi], s_dig[fi], stk, s_Q, s_inv, bj, s_Sk, s_lam); break;
    case 4: small_column<R, D, M, KIDX, 4>(a, buf, pi * 4, s_fbk[fi], s_dig[fi], stk, s_Q, s_inv, bj, s_Sk, s_lam); break;
    default: small_column<R, D, M, KIDX, 8>(a, buf, pi * 8, s_fbk[fi], s_dig[fi], stk, s_Q, s_inv, bj, s_Sk, s_lam); break;
    }
  }
  __syncthreads();
  other_stages(false);
  for (int c = warp; c < nc; c += kSmallThreads / 32)
  {
    int64_t const gb = int64_t(s_cell[c]) * TS;
    const R *bc      = buf + c * TS;
    for (int i = lane; i < TS; i += 32)
    {
      if (out64)
      {
        out64[gb + i] = double(bc[i]);
        if (zcopy)
          zcopy[gb + i] = float(bc[i]);
      }
      else
        outR[gb + i] = bc[i];
    }
  }
}

template<typename R>
struct line_tables
{
  R *Q = nullptr, *QT = nullptr, *theta = nullptr, *self = nullptr;
  ~line_tables()
  {
    cudaFree(Q);
    cudaFree(QT);
    cudaFree(theta);
    cudaFree(self);
  }
};

struct line_factor
{
  int k = 0;
  int nunits = 0;   // (pencil, group range) units of the larger pencils
  int max_rows = 0; // largest Rp * G of its units (shared memory)
  int max_rp   = 0; // largest padded pencil size (matrix tiles)
  int nbatches = 0; // batches of pencils of 1, 2, 4 or 8 cells
  int4 *units = nullptr, *batches = nullptr, *bcells = nullptr;
  int *pen_off = nullptr, *pen_m = nullptr, *pen_tab = nullptr, *pen_cells = nullptr;
  ~line_factor()
  {
    cudaFree(units);
    cudaFree(batches);
    cudaFree(bcells);
    cudaFree(pen_off);
    cudaFree(pen_m);
    cudaFree(pen_tab);
    cudaFree(pen_cells);
  }
};

template<typename T>
int upload(T **dst, std::vector<T> const &src, int64_t &bytes)
{
  size_t const b = sizeof(T) * std::max<size_t>(src.size(), 1);
  ASGK_CUDA(cudaMalloc(dst, b));
  if (!src.empty())
    ASGK_CUDA(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(),
                         cudaMemcpyHostToDevice));
  bytes += int64_t(b);
  return ASGK_OK;
}
} // namespace

struct line_data
{
  int d = 0, rows = 0, ts = 0, r1 = 0, m = 0;
  int line[3] = {0, 0, 0};
  int nonline[6] = {0, 0, 0, 0, 0, 0};
  double shift = 1, dt = 0;
  int *c1 = nullptr, *tab_off = nullptr, *tab_th = nullptr, *tab_rp = nullptr;
  line_tables<double> t64;
  line_tables<float> t32;
  std::vector<std::unique_ptr<line_factor>> factors;
  double *work = nullptr; // two intermediate vectors (rows * ts doubles each)
  // a factor's small-pencil and larger-pencil launches touch disjoint cells:
  // the larger ones run on a second stream, forked from and joined back to
  // the caller's (parallel branches when the caller records a graph)
  cudaStream_t side = nullptr;
  cudaEvent_t fork[3] = {nullptr, nullptr, nullptr}, join[3] = {nullptr, nullptr, nullptr};
  ~line_data()
  {
    for (int q = 0; q < 3; q++)
    {
      if (fork[q])
        cudaEventDestroy(fork[q]);
      if (join[q])
        cudaEventDestroy(join[q]);
    }
    if (side)
      cudaStreamDestroy(side);
    cudaFree(c1);
    cudaFree(tab_off);
    cudaFree(tab_th);
    cudaFree(tab_rp);
    cudaFree(work);
  }
};

void line_free(line_data *ld) { delete ld; }

int line_build(plan_data const &p, double dt, line_data **out, int64_t &bytes)
{
  *out = nullptr;
  if (!p.global || p.gchains > 0 || p.n != 3 || p.rows != p.cols)
    return ASGK_ERR_UNSUPPORTED;
  int const d         = p.d;
  int64_t const nconn = int64_t(p.g_conn_row.size());
  int r1              = 0;
  for (int64_t j = 0; j < nconn; j++)
    r1 = std::max(r1, std::max(p.g_conn_row[j], p.g_conn_col[j]) + 1);
  std::vector<double> B(size_t(nconn) * d * 10);
  ASGK_CUDA(cudaMemcpy(B.data(), p.gB64, sizeof(double) * B.size(),
                       cudaMemcpyDeviceToHost));
  // the full 1D operator of every dimension (3 r1 square, row-major)
  int const nf = 3 * r1;
  std::vector<std::vector<double>> F(d, std::vector<double>(size_t(nf) * nf, 0.0));
  for (int64_t j = 0; j < nconn; j++)
    for (int k = 0; k < d; k++)
    {
      const double *b = &B[size_t(j * d + k) * 10];
      int const r = p.g_conn_row[j], c = p.g_conn_col[j];
      for (int jj = 0; jj < 3; jj++)
        for (int i = 0; i < 3; i++)
          F[k][size_t(3 * r + i) * nf + 3 * c + jj] = b[i + 3 * jj];
    }
  // line dimensions: nonzero symmetric operators
  std::vector<int> line, nonline;
  for (int k = 0; k < d; k++)
  {
    double mx = 0, asym = 0;
    for (int r = 0; r < nf; r++)
      for (int c = 0; c < nf; c++)
      {
        mx   = std::max(mx, std::abs(F[k][size_t(r) * nf + c]));
        asym = std::max(asym, std::abs(F[k][size_t(r) * nf + c] - F[k][size_t(c) * nf + r]));
      }
    if (mx > 0 && asym <= 1e-12 * mx)
      line.push_back(k);
    else
      nonline.push_back(k);
  }
  if (line.empty() || line.size() > 3)
    return ASGK_ERR_UNSUPPORTED;
  int const M = int(line.size());
  auto ld     = std::make_unique<line_data>();
  ld->d = d, ld->rows = p.rows, ld->ts = p.tensor, ld->r1 = r1, ld->m = M, ld->dt = dt;
  ld->shift = 1.0 - dt * p.g_identity;
  for (int q = 0; q < M; q++)
    ld->line[q] = line[q];
  for (size_t q = 0; q < nonline.size(); q++)
    ld->nonline[q] = nonline[q];
  // every cell's 1D cells (its self connections in the global plan's
  // diagonal pair list)
  std::vector<int> selfc(size_t(p.rows) * d), c1(size_t(p.rows) * d);
  ASGK_CUDA(cudaMemcpy(selfc.data(), p.idx, sizeof(int) * selfc.size(),
                       cudaMemcpyDeviceToHost));
  for (size_t e = 0; e < selfc.size(); e++)
    c1[e] = p.g_conn_row[selfc[e]];
  // self blocks of the line dimensions and their eigendecompositions
  std::vector<double> self(size_t(M) * r1 * kSelfEntry, 0.0);
  for (int q = 0; q < M; q++)
    for (int c = 0; c < r1; c++)
    {
      std::vector<double> S(9), V, w;
      for (int i = 0; i < 3; i++)
        for (int jj = 0; jj < 3; jj++)
          S[size_t(i) * 3 + jj] = F[line[q]][size_t(3 * c + i) * nf + 3 * c + jj];
      if (!sym_eig(3, S, V, w))
        return ASGK_ERR_UNSUPPORTED;
      double *e = &self[(size_t(q) * r1 + c) * kSelfEntry];
      for (int i = 0; i < 3; i++)
        for (int jj = 0; jj < 3; jj++)
        {
          e[i + 3 * jj]      = V[size_t(i) * 3 + jj]; // P(i, jj), column jj eigenvector
          e[12 + i + 3 * jj] = S[size_t(i) * 3 + jj];
        }
      for (int i = 0; i < 3; i++)
        e[9 + i] = w[i];
    }
  // pencils of every line dimension, their matrices by (operator, 1D set)
  int bits = 1;
  while ((1 << bits) < r1)
    ++bits;
  if (bits * (d - 1) > 63)
    return ASGK_ERR_UNSUPPORTED;
  std::vector<int> opid(M);
  for (int q = 0; q < M; q++)
  {
    opid[q] = q;
    for (int q2 = 0; q2 < q; q2++)
      if (F[line[q2]] == F[line[q]])
      {
        opid[q] = opid[q2];
        break;
      }
  }
  std::map<std::pair<int, std::vector<int>>, int> tabs;
  std::vector<double> Qh, QTh, thh;
  std::vector<int> toff, tth, trp;
  int const ng = ipow3l(d - M);
  for (int q = 0; q < M; q++)
  {
    int const k = line[q];
    std::vector<std::pair<uint64_t, int>> keyed(p.rows);
    for (int c = 0; c < p.rows; c++)
    {
      uint64_t key = 0;
      for (int j = 0; j < d; j++)
        if (j != k)
          key = (key << bits) | uint64_t(c1[size_t(c) * d + j]);
      keyed[c] = {key, c};
    }
    std::sort(keyed.begin(), keyed.end(), [&](auto const &x, auto const &y) {
      if (x.first != y.first)
        return x.first < y.first;
      return c1[size_t(x.second) * d + k] < c1[size_t(y.second) * d + k];
    });
    std::vector<int> pen_off, pen_m, pen_tab, pen_cells;
    for (size_t s = 0; s < keyed.size();)
    {
      size_t e = s;
      while (e < keyed.size() && keyed[e].first == keyed[s].first)
        ++e;
      std::vector<int> set;
      pen_off.push_back(int(pen_cells.size()));
      for (size_t i = s; i < e; i++)
      {
        pen_cells.push_back(keyed[i].second);
        set.push_back(c1[size_t(keyed[i].second) * d + k]);
      }
      pen_m.push_back(int(e - s));
      auto const tk = std::make_pair(opid[q], set);
      auto it       = tabs.find(tk);
      if (it == tabs.end())
      {
        int const Rr = 3 * int(set.size());
        int const Rp = (Rr + 3) / 4 * 4;
        std::vector<double> A(size_t(Rr) * Rr);
        for (int a2 = 0; a2 < Rr; a2++)
          for (int b2 = 0; b2 < Rr; b2++)
            A[size_t(a2) * Rr + b2] =
                F[k][size_t(3 * set[a2 / 3] + a2 % 3) * nf + 3 * set[b2 / 3] + b2 % 3];
        std::vector<double> V, w;
        if (!sym_eig(Rr, A, V, w))
          return ASGK_ERR_UNSUPPORTED;
        int const id = int(toff.size());
        toff.push_back(int(Qh.size()));
        trp.push_back(Rp);
        // Q [t][r] = eigenvector r's entry t; QT [r][t] = the same; theta
        // padded to Rp entries
        Qh.resize(Qh.size() + size_t(Rr) * Rp, 0.0);
        QTh.resize(QTh.size() + size_t(Rr) * Rp, 0.0);
        double *Qt = &Qh[toff.back()], *QTt = &QTh[toff.back()];
        for (int t = 0; t < Rr; t++)
          for (int r = 0; r < Rr; r++)
          {
            Qt[size_t(t) * Rp + r]  = V[size_t(t) * Rr + r];
            QTt[size_t(r) * Rp + t] = V[size_t(t) * Rr + r];
          }
        tth.push_back(int(thh.size()));
        thh.resize(thh.size() + Rp, 0.0);
        for (int r = 0; r < Rr; r++)
          thh[tth.back() + r] = w[r];
        it = tabs.emplace(tk, id).first;
      }
      pen_tab.push_back(it->second);
      s = e;
    }
    // pencils ordered by size (larger first), then by matrix; pencils of
    // 1, 2, 4 or 8 cells go in batches of up to kSmallCells cells of one
    // matrix (k_line_small), the others are cut into group-range units
    {
      std::vector<int> order(pen_m.size());
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        if (pen_m[x] != pen_m[y])
          return pen_m[x] > pen_m[y];
        return pen_tab[x] < pen_tab[y];
      });
      std::vector<int> o_off, o_m, o_tab;
      for (int pe : order)
      {
        o_off.push_back(pen_off[pe]);
        o_m.push_back(pen_m[pe]);
        o_tab.push_back(pen_tab[pe]);
      }
      pen_off.swap(o_off);
      pen_m.swap(o_m);
      pen_tab.swap(o_tab);
    }
    auto small = [](int m) { return m == 1 || m == 2 || m == 4 || m == kSmallMaxM; };
    int rpmax = 0;
    for (size_t pe = 0; pe < pen_m.size(); pe++)
      if (!small(pen_m[pe]))
        rpmax = std::max(rpmax, trp[pen_tab[pe]]);
    // a unit's (4-row block, group) items: at most two per item slot; its
    // rows x groups bound its shared memory
    int const budget = std::max(rpmax, 4 * kLineItems);
    int max_rp       = 0;
    std::vector<int4> units, batches, bcells;
    int max_rows = 0;
    for (size_t pe = 0; pe < pen_m.size();)
    {
      int const m = pen_m[pe];
      if (small(m))
      {
        int const per = kSmallCells / m;
        size_t e      = pe;
        while (e < pen_m.size() && e - pe < size_t(per) && pen_m[e] == m &&
               pen_tab[e] == pen_tab[pe])
          ++e;
        int const tb = pen_tab[pe];
        batches.push_back(make_int4(int(e - pe), m, toff[tb], tth[tb]));
        for (size_t p2 = pe; p2 < e; p2++)
          for (int i = 0; i < m; i++)
          {
            int const cell = pen_cells[pen_off[p2] + i];
            int so[3]      = {0, 0, 0};
            for (int q2 = 0; q2 < M; q2++)
              so[q2] = (q2 * r1 + c1[size_t(cell) * d + line[q2]]) * kSelfEntry;
            bcells.push_back(make_int4(cell, so[0], so[1], so[2]));
          }
        while (bcells.size() % kSmallCells)
          bcells.push_back(make_int4(0, 0, 0, 0));
        pe = e;
        continue;
      }
      int const Rp = trp[pen_tab[pe]];
      int const G  = std::max(1, std::min(std::min(ng, 27), budget / Rp));
      max_rp       = std::max(max_rp, Rp);
      for (int g0 = 0; g0 < ng; g0 += G)
      {
        int const gc = std::min(G, ng - g0);
        units.push_back(make_int4(int(pe), g0, gc, 0));
        max_rows = std::max(max_rows, Rp * gc);
      }
      ++pe;
    }
    auto fac      = std::make_unique<line_factor>();
    fac->k        = k;
    fac->nunits   = int(units.size());
    fac->max_rows = max_rows;
    fac->max_rp   = max_rp;
    fac->nbatches = int(batches.size());
    int rc;
    if ((rc = upload(&fac->units, units, bytes)) || (rc = upload(&fac->batches, batches, bytes)) ||
        (rc = upload(&fac->bcells, bcells, bytes)) ||
        (rc = upload(&fac->pen_off, pen_off, bytes)) ||
        (rc = upload(&fac->pen_m, pen_m, bytes)) || (rc = upload(&fac->pen_tab, pen_tab, bytes)) ||
        (rc = upload(&fac->pen_cells, pen_cells, bytes)))
      return rc;
    ld->factors.push_back(std::move(fac));
  }
  std::vector<float> Q32(Qh.begin(), Qh.end()), QT32(QTh.begin(), QTh.end()),
      th32(thh.begin(), thh.end()), self32(self.begin(), self.end());
  int rc;
  if ((rc = upload(&ld->c1, c1, bytes)) || (rc = upload(&ld->tab_off, toff, bytes)) ||
      (rc = upload(&ld->tab_th, tth, bytes)) || (rc = upload(&ld->tab_rp, trp, bytes)) || (rc = upload(&ld->t64.Q, Qh, bytes)) ||
      (rc = upload(&ld->t64.QT, QTh, bytes)) || (rc = upload(&ld->t64.theta, thh, bytes)) ||
      (rc = upload(&ld->t64.self, self, bytes)) || (rc = upload(&ld->t32.Q, Q32, bytes)) ||
      (rc = upload(&ld->t32.QT, QT32, bytes)) || (rc = upload(&ld->t32.theta, th32, bytes)) ||
      (rc = upload(&ld->t32.self, self32, bytes)))
    return rc;
  size_t const wb = sizeof(double) * 2 * size_t(p.rows) * p.tensor;
  ASGK_CUDA(cudaMalloc(&ld->work, wb));
  ASGK_CUDA(cudaStreamCreateWithFlags(&ld->side, cudaStreamNonBlocking));
  for (int q = 0; q < M; q++)
  {
    ASGK_CUDA(cudaEventCreateWithFlags(&ld->fork[q], cudaEventDisableTiming));
    ASGK_CUDA(cudaEventCreateWithFlags(&ld->join[q], cudaEventDisableTiming));
  }
  bytes += int64_t(wb);
  *out = ld.release();
  return ASGK_OK;
}

namespace
{
template<typename R, int D, int M, int KIDX>
int launch_factor(line_data const &ld, line_factor const &f, const double *in64,
                  const R *inR, double *out64, R *outR, bool bj,
                  const double *sc, double *vscale, float *vc, float *zc,
                  cudaStream_t s)
{
  constexpr int NC  = ipow3l(M - 1);
  constexpr int NCP = NC == 1 ? 1 : (NC == 3 ? 4 : 12);
  line_tables<R> const &t = [&]() -> line_tables<R> const & {
    if constexpr (sizeof(R) == 8)
      return ld.t64;
    else
      return ld.t32;
  }();
  line_args<R> a{};
  a.units = f.units, a.pen_off = f.pen_off, a.pen_m = f.pen_m, a.pen_tab = f.pen_tab;
  a.pen_cells = f.pen_cells, a.c1 = ld.c1, a.tab_off = ld.tab_off, a.tab_th = ld.tab_th;
  a.tab_rp = ld.tab_rp;
  a.Q = t.Q, a.QT = t.QT, a.theta = t.theta, a.self = t.self, a.r1 = ld.r1;
  a.k = f.k, a.kidx = KIDX;
  for (int i = 0; i < 3; i++)
    a.line[i] = ld.line[i];
  for (int i = 0; i < 6; i++)
    a.nonline[i] = ld.nonline[i];
  a.shift = R(ld.shift), a.dt = R(ld.dt);
  a.st_k = ipow3l(D - 1 - f.k);
  for (int q = 0; q < 3; q++)
    a.st_line[q] = q < M ? ipow3l(D - 1 - ld.line[q]) : 0;
  bool const both = f.nbatches > 0 && f.nunits > 0;
  cudaStream_t sb = s;
  if (both)
  {
    sb = ld.side;
    ASGK_CUDA(cudaEventRecord(ld.fork[KIDX], s));
    ASGK_CUDA(cudaStreamWaitEvent(sb, ld.fork[KIDX], 0));
  }
  if (f.nunits > 0)
  {
    // the (member, group) tables (members x groups <= max_rows / 3), X, Y and
    // the matrix tiles
    size_t const shm = ((12 * (size_t(f.max_rows) / 3 + 1) + 15) / 16) * 16 +
                       sizeof(R) * (2 * size_t(f.max_rows) * NCP +
                                    2 * size_t(kLineTile) * f.max_rp);
    auto kern        = k_line_factor<R, D, M, KIDX>;
    ASGK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(shm)));
    kern<<<f.nunits, kLineThreads, shm, sb>>>(a, in64, inR, out64, outR, bj ? 1 : 0,
                                              sc, vscale, vc, zc, g_gate);
    ASGK_LAUNCHED();
  }
  if (f.nbatches > 0)
  {
    size_t const shm = sizeof(R) * size_t(kSmallCells) * ipow3l(D);
    auto kern        = k_line_small<R, D, M, KIDX>;
    ASGK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(shm)));
    kern<<<f.nbatches, kSmallThreads, shm, s>>>(a, f.batches, f.bcells, in64, inR, out64,
                                                outR, bj ? 1 : 0, sc, vscale, vc, zc, g_gate);
    ASGK_LAUNCHED();
  }
  if (both)
  {
    ASGK_CUDA(cudaEventRecord(ld.join[KIDX], sb));
    ASGK_CUDA(cudaStreamWaitEvent(s, ld.join[KIDX], 0));
  }
  return ASGK_OK;
}

template<typename R, int D, int M, int KIDX>
int factor_q(line_data const &ld, const double *in64, const R *inR, double *out64,
             R *outR, bool bj, const double *sc, double *vscale, float *vc,
             float *zc, cudaStream_t s)
{
  return launch_factor<R, D, M, KIDX>(ld, *ld.factors[KIDX], in64, inR, out64, outR,
                                      bj, sc, vscale, vc, zc, s);
}

template<typename R, int D, int M>
int apply_dm(line_data const &ld, double *v, double *z, const double *sc,
             float *vc, float *zc, cudaStream_t s)
{
  int64_t const n = int64_t(ld.rows) * ld.ts;
  R *w0 = reinterpret_cast<R *>(ld.work);
  R *w1 = w0 + n;
  R *cur = nullptr;
  for (int q = 0; q < M; q++)
  {
    bool const first = q == 0, last = q == M - 1;
    R *dst = (q % 2 == 0) ? w0 : w1;
    const double *i64 = first ? v : nullptr;
    const R *iR       = first ? nullptr : cur;
    double *o64       = last ? z : nullptr;
    R *oR             = last ? nullptr : dst;
    const double *fsc = first ? sc : nullptr;
    double *fvs       = first && sc ? v : nullptr;
    float *fvc        = first ? vc : nullptr;
    float *lzc        = last ? zc : nullptr;
    int rc            = ASGK_ERR_UNSUPPORTED;
    if (q == 0)
      rc = factor_q<R, D, M, 0>(ld, i64, iR, o64, oR, !first, fsc, fvs, fvc, lzc, s);
    else if constexpr (M >= 2)
    {
      if (q == 1)
        rc = factor_q<R, D, M, 1>(ld, i64, iR, o64, oR, !first, fsc, fvs, fvc, lzc, s);
      else if constexpr (M >= 3)
        rc = factor_q<R, D, M, 2>(ld, i64, iR, o64, oR, !first, fsc, fvs, fvc, lzc, s);
    }
    if (rc)
      return rc;
    cur = dst;
  }
  return ASGK_OK;
}

template<typename R, int D>
int apply_d(line_data const &ld, double *v, double *z, const double *sc,
            float *vc, float *zc, cudaStream_t s)
{
  switch (ld.m)
  {
  case 1: return apply_dm<R, D, 1>(ld, v, z, sc, vc, zc, s);
  case 2:
    if constexpr (D >= 2)
      return apply_dm<R, D, 2>(ld, v, z, sc, vc, zc, s);
    break;
  case 3:
    if constexpr (D >= 3)
      return apply_dm<R, D, 3>(ld, v, z, sc, vc, zc, s);
    break;
  default: break;
  }
  return ASGK_ERR_UNSUPPORTED;
}
} // namespace

int line_apply(line_data const &ld, bool low, double *v, double *z,
               const double *scale_state, float *vcopy, float *zcopy,
               cudaStream_t s)
{
  auto go = [&](auto tag) -> int {
    using R = decltype(tag);
    switch (ld.d)
    {
    case 1: return apply_d<R, 1>(ld, v, z, scale_state, vcopy, zcopy, s);
    case 2: return apply_d<R, 2>(ld, v, z, scale_state, vcopy, zcopy, s);
    case 3: return apply_d<R, 3>(ld, v, z, scale_state, vcopy, zcopy, s);
    case 4: return apply_d<R, 4>(ld, v, z, scale_state, vcopy, zcopy, s);
    case 5: return apply_d<R, 5>(ld, v, z, scale_state, vcopy, zcopy, s);
    case 6: return apply_d<R, 6>(ld, v, z, scale_state, vcopy, zcopy, s);
    default: return ASGK_ERR_UNSUPPORTED;
    }
  };
  return low ? go(float{}) : go(double{});
}

int line_info(line_data const &ld, int *dims)
{
  for (int q = 0; q < ld.m; q++)
    dims[q] = ld.line[q];
  return ld.m;
}

} // namespace asgk
