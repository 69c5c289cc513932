// Learned preconditioner: a per-cell MLP trained and run on the GPU.
//
// Network: f(u) = W4 g(W3 g(W2 g(W1 u + b1) + b2) + b3) + b4, g = GELU (erf
// form), layer widths in -> H -> H -> H -> out with in = n^d + d (the cell's
// residual block scaled to unit norm, then its d levels / max level) and
// out = n^d.  As a preconditioner z = M(v) applies f cell by cell:
//   z_c = ||v_c|| * f([v_c / ||v_c||, levels_c / L]),
// which makes M positively homogeneous (M(a v) = a M(v), a > 0).
//
// GEMMs run on the tensor cores in BF16 with FP32 accumulation
// (mma.sync.m16n8k16), bias/GELU fused into their epilogues; FP32 master
// weights with Adam; MSE loss on scaled targets.
#include "mlp.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

namespace asgk
{
namespace
{
using bf16 = __nv_bfloat16;

constexpr int kLayers = 4;

// --------------------------------------------------------------- GEMM
// C[M, N] = op(A)[M, K] * op(B)[K, N] with BF16 operands, FP32 accumulation.
// op(A) = A (row-major M x K, lda) or A^T (A stored K x M); op(B) = B
// (row-major K x N, ldb) or B^T (B stored N x K).  64 x 64 x 32 tiles, 4
// warps of 32 x 32, operands staged in shared memory ([m][k] and [k][n]).
enum epilogue : int
{
  EPI_STORE_F32   = 0, // C = acc  (or C += acc when accumulate)
  EPI_BIAS_GELU   = 1, // pre = acc + bias (f32); out = gelu(pre) (bf16)
  EPI_BIAS_F32    = 2, // C = acc + bias (f32)
  EPI_DGELU       = 3  // out = acc * gelu'(pre) (bf16)
};

constexpr int TM = 64, TN = 64, TK = 32;

__device__ __forceinline__ float gelu(float x)
{
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float dgelu(float x)
{
  float const cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  float const pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi)
{
  uint32_t const l = __bfloat16_as_ushort(lo);
  uint32_t const h = __bfloat16_as_ushort(hi);
  return l | (h << 16);
}

__device__ __forceinline__ void mma16816(float (&c)[4], uint32_t const (&a)[4],
                                         uint32_t const (&b)[2])
{
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template<bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(128)
    k_gemm(int M, int N, int K, const bf16 *__restrict__ A, int lda,
           const bf16 *__restrict__ B, int ldb, float *__restrict__ C,
           int ldc, const float *__restrict__ bias,
           const float *__restrict__ pre_in, float *__restrict__ pre_out,
           bf16 *__restrict__ out, int ldo, int accumulate)
{
  __shared__ bf16 As[TM][TK + 8];
  __shared__ bf16 Bs[TK][TN + 8];
  int const m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  int const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int const wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  int const g = lane >> 2, tg = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 4; e++)
        acc[i][j][e] = 0.f;

  bf16 const zero = __float2bfloat16(0.f);
  for (int k0 = 0; k0 < K; k0 += TK)
  {
    // stage op(A)[m0:m0+64, k0:k0+32] and op(B)[k0:k0+32, n0:n0+64]
    for (int i = tid; i < TM * TK; i += 128)
    {
      int const mm = TA ? (i % TM) : (i / TK), kk = TA ? (i / TM) : (i % TK);
      int const gm = m0 + mm, gk = k0 + kk;
      bf16 v = zero;
      if (gm < M && gk < K)
        v = TA ? A[int64_t(gk) * lda + gm] : A[int64_t(gm) * lda + gk];
      As[mm][kk] = v;
    }
    for (int i = tid; i < TK * TN; i += 128)
    {
      int const kk = TB ? (i % TK) : (i / TN), nn = TB ? (i / TK) : (i % TN);
      int const gk = k0 + kk, gn = n0 + nn;
      bf16 v = zero;
      if (gk < K && gn < N)
        v = TB ? B[int64_t(gn) * ldb + gk] : B[int64_t(gk) * ldb + gn];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < TK; ks += 16)
    {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; i++)
      {
        int const r = wm + i * 16 + g, c = ks + tg * 2;
        af[i][0] = pack2(As[r][c], As[r][c + 1]);
        af[i][1] = pack2(As[r + 8][c], As[r + 8][c + 1]);
        af[i][2] = pack2(As[r][c + 8], As[r][c + 9]);
        af[i][3] = pack2(As[r + 8][c + 8], As[r + 8][c + 9]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
      {
        int const n = wn + j * 8 + g, k = ks + tg * 2;
        bfr[j][0] = pack2(Bs[k][n], Bs[k + 1][n]);
        bfr[j][1] = pack2(Bs[k + 8][n], Bs[k + 9][n]);
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
          mma16816(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
  // epilogue: element (r, c) of every accumulator fragment
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 4; e++)
      {
        int const r = m0 + wm + i * 16 + g + ((e >= 2) ? 8 : 0);
        int const c = n0 + wn + j * 8 + tg * 2 + (e & 1);
        if (r >= M || c >= N)
          continue;
        float const v = acc[i][j][e];
        if constexpr (EPI == EPI_STORE_F32)
        {
          float *dst = C + int64_t(r) * ldc + c;
          *dst       = accumulate ? (*dst + v) : v;
        }
        else if constexpr (EPI == EPI_BIAS_F32)
          C[int64_t(r) * ldc + c] = v + bias[c];
        else if constexpr (EPI == EPI_BIAS_GELU)
        {
          float const p = v + bias[c];
          if (pre_out)
            pre_out[int64_t(r) * ldo + c] = p;
          out[int64_t(r) * ldo + c] = __float2bfloat16(gelu(p));
        }
        else // EPI_DGELU
          out[int64_t(r) * ldo + c] =
              __float2bfloat16(v * dgelu(pre_in[int64_t(r) * ldo + c]));
      }
}

template<bool TA, bool TB, int EPI>
int gemm(int M, int N, int K, const bf16 *A, int lda, const bf16 *B, int ldb,
         float *C, int ldc, const float *bias, const float *pre_in,
         float *pre_out, bf16 *out, int ldo, int accumulate, cudaStream_t s)
{
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  k_gemm<TA, TB, EPI><<<grid, 128, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc,
                                           bias, pre_in, pre_out, out, ldo,
                                           accumulate);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

// ------------------------------------------------------------ small kernels

__global__ void k_f32_to_bf16(const float *__restrict__ a, bf16 *__restrict__ b,
                              int64_t n)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    b[i] = __float2bfloat16(a[i]);
}

// column sums of a row-major (rows x cols) bf16 matrix -> out (f32)
__global__ void k_colsum(const bf16 *__restrict__ a, int rows, int cols,
                         float *__restrict__ out)
{
  int const c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols)
    return;
  float s = 0.f;
  for (int r = 0; r < rows; r++)
    s += __bfloat162float(a[int64_t(r) * cols + c]);
  out[c] = s;
}

// dY = (Y - T) * scale as bf16; partial sums of (Y - T)^2 per block
__global__ void k_mse_grad(const float *__restrict__ y,
                           const float *__restrict__ t, int64_t n, float scale,
                           bf16 *__restrict__ dy, float *__restrict__ part)
{
  __shared__ float sh[256];
  float s = 0.f;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    float const d = y[i] - t[i];
    dy[i]         = __float2bfloat16(d * scale);
    s += d * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1)
  {
    if (threadIdx.x < o)
      sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    part[blockIdx.x] = sh[0];
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, int64_t n,
                       float lr, float b1, float b2, float eps, float bc1,
                       float bc2)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    float const gi = g[i];
    float const mi = b1 * m[i] + (1.f - b1) * gi;
    float const vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i]           = mi;
    v[i]           = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// Preconditioner input rows: one row per cell, [v_c / s_c, levels / L, 0...]
// with s_c = ||v_c||_2 (1 when v_c = 0); s stored for the output scaling.
__global__ void k_pc_features(const double *__restrict__ v, int cells, int ts,
                              int d, const float *__restrict__ lev, int ldx,
                              bf16 *__restrict__ X, double *__restrict__ s)
{
  int const c    = blockIdx.x;
  const double *vc = v + int64_t(c) * ts;
  __shared__ double sh[256];
  double acc = 0;
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
    acc += vc[i] * vc[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1)
  {
    if (threadIdx.x < o)
      sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  double const nrm = sqrt(sh[0]);
  double const sc  = (nrm > 0) ? nrm : 1.0;
  bf16 *row        = X + int64_t(c) * ldx;
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
    row[i] = __float2bfloat16(float(vc[i] / sc));
  for (int i = threadIdx.x; i < d; i += blockDim.x)
    row[ts + i] = __float2bfloat16(lev[int64_t(c) * d + i]);
  if (threadIdx.x == 0)
    s[c] = (nrm > 0) ? nrm : 0.0;
}

// z_c = s_c * y_c
__global__ void k_pc_output(const float *__restrict__ y, int cells, int ts,
                            const double *__restrict__ s,
                            double *__restrict__ z)
{
  int64_t const n = int64_t(cells) * ts;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    z[i] = s[i / ts] * double(y[i]);
}

// Training rows from (v, e) cell pairs: X = [v_c/s_c, lev], T = e_c/s_c.
__global__ void k_train_rows(const double *__restrict__ v,
                             const double *__restrict__ e,
                             const int *__restrict__ cell_of_row,
                             const int *__restrict__ sample_of_row, int rows,
                             int ts, int d, int64_t stride,
                             const float *__restrict__ lev, int ldx,
                             bf16 *__restrict__ X, float *__restrict__ T)
{
  int const r = blockIdx.x;
  if (r >= rows)
    return;
  int const c        = cell_of_row[r];
  int64_t const base = int64_t(sample_of_row[r]) * stride + int64_t(c) * ts;
  __shared__ double sh[256];
  double acc = 0;
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
    acc += v[base + i] * v[base + i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1)
  {
    if (threadIdx.x < o)
      sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  double const nrm = sqrt(sh[0]);
  double const sc  = (nrm > 0) ? nrm : 1.0;
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
  {
    X[int64_t(r) * ldx + i] = __float2bfloat16(float(v[base + i] / sc));
    T[int64_t(r) * ts + i]  = float(e[base + i] / sc);
  }
  for (int i = threadIdx.x; i < d; i += blockDim.x)
    X[int64_t(r) * ldx + ts + i] = __float2bfloat16(lev[int64_t(c) * d + i]);
}

int grid1(int64_t n) { return int(std::min<int64_t>(1024, (n + 255) / 256)); }

} // namespace

// Device-resident network and its training state.
struct mlp_state
{
  int d = 0, ts = 0, in = 0, ldx = 0, hidden = 0, cells = 0;
  int dims[kLayers + 1] = {};
  float *W[kLayers] = {}, *b[kLayers] = {};          // masters (row-major in x out)
  bf16 *Wb[kLayers] = {};                              // bf16 copies
  float *gW[kLayers] = {}, *gb[kLayers] = {};
  float *mW[kLayers] = {}, *vW[kLayers] = {}, *mb[kLayers] = {}, *vb[kLayers] = {};
  float *lev = nullptr;                                // cells x d
  // activations for up to cap rows
  int cap = 0;
  bf16 *X = nullptr;
  float *pre[kLayers - 1] = {};
  bf16 *h[kLayers - 1] = {};
  float *Y = nullptr, *T = nullptr, *part = nullptr;
  bf16 *dY = nullptr, *dP[kLayers - 1] = {}, *dH = nullptr;
  double *scale = nullptr;
  int64_t step = 0;
  std::vector<void *> owned;

  template<typename P>
  int alloc(P **p, int64_t n)
  {
    *p = nullptr;
    if (n <= 0)
      return ASGK_OK;
    if (cudaMalloc(reinterpret_cast<void **>(p), sizeof(P) * n) != cudaSuccess)
    {
      cudaGetLastError();
      return ASGK_ERR_ALLOC;
    }
    owned.push_back(*p);
    return ASGK_OK;
  }
  ~mlp_state()
  {
    for (void *p : owned)
      cudaFree(p);
  }
  int ensure_rows(int rows)
  {
    if (rows <= cap)
      return ASGK_OK;
    // activations are reallocated (old buffers stay owned until destroy)
    int rc;
    if ((rc = alloc(&X, int64_t(rows) * ldx)) || (rc = alloc(&Y, int64_t(rows) * ts)) ||
        (rc = alloc(&T, int64_t(rows) * ts)) || (rc = alloc(&dY, int64_t(rows) * ts)) ||
        (rc = alloc(&dH, int64_t(rows) * hidden)) || (rc = alloc(&part, 1024)) ||
        (rc = alloc(&scale, rows)))
      return rc;
    for (int l = 0; l < kLayers - 1; l++)
      if ((rc = alloc(&pre[l], int64_t(rows) * hidden)) ||
          (rc = alloc(&h[l], int64_t(rows) * hidden)) ||
          (rc = alloc(&dP[l], int64_t(rows) * hidden)))
        return rc;
    cudaMemset(X, 0, sizeof(bf16) * int64_t(rows) * ldx);
    cap = rows;
    return ASGK_OK;
  }
  int sync_bf16(cudaStream_t s)
  {
    for (int l = 0; l < kLayers; l++)
    {
      int64_t const n = int64_t(dims[l]) * dims[l + 1];
      k_f32_to_bf16<<<grid1(n), 256, 0, s>>>(W[l], Wb[l], n);
      ASGK_LAUNCHED();
    }
    return ASGK_OK;
  }
  // forward pass on rows [0, rows) of X; keeps pre-activations for training
  int forward(int rows, cudaStream_t s)
  {
    const bf16 *in_act = X;
    int in_ld          = ldx;
    for (int l = 0; l < kLayers - 1; l++)
    {
      if (int rc = gemm<false, false, EPI_BIAS_GELU>(
              rows, hidden, dims[l], in_act, in_ld, Wb[l], dims[l + 1],
              nullptr, 0, b[l], nullptr, pre[l], h[l], hidden, 0, s))
        return rc;
      in_act = h[l];
      in_ld  = hidden;
    }
    return gemm<false, false, EPI_BIAS_F32>(rows, ts, hidden, in_act, in_ld,
                                             Wb[kLayers - 1], ts, Y, ts,
                                             b[kLayers - 1], nullptr, nullptr,
                                             nullptr, 0, 0, s);
  }
  // gradients of 0.5 * sum((Y - T)^2) * gscale w.r.t. all weights
  int backward(int rows, float gscale, double *loss, cudaStream_t s)
  {
    int64_t const n = int64_t(rows) * ts;
    int const gb1   = grid1(n);
    k_mse_grad<<<gb1, 256, 0, s>>>(Y, T, n, gscale, dY, part);
    ASGK_LAUNCHED();
    // layer 4: dW4 = h3^T dY, db4 = colsum(dY), dH = dY W4^T
    const bf16 *dcur = dY;
    int dcols        = ts;
    for (int l = kLayers - 1; l >= 0; l--)
    {
      const bf16 *act = (l == 0) ? X : h[l - 1];
      int const act_ld = (l == 0) ? ldx : hidden;
      int const kin    = dims[l];
      if (int rc = gemm<true, false, EPI_STORE_F32>(
              kin, dcols, rows, act, act_ld, dcur, dcols, gW[l], dcols,
              nullptr, nullptr, nullptr, nullptr, 0, 0, s))
        return rc;
      k_colsum<<<(dcols + 127) / 128, 128, 0, s>>>(dcur, rows, dcols, gb[l]);
      ASGK_LAUNCHED();
      if (l == 0)
        break;
      // dH = dcur W_l^T, then dP = dH * gelu'(pre_{l-1})
      if (int rc = gemm<false, true, EPI_DGELU>(
              rows, hidden, dcols, dcur, dcols, Wb[l], dcols, nullptr, 0,
              nullptr, pre[l - 1], nullptr, dP[l - 1], hidden, 0, s))
        return rc;
      dcur  = dP[l - 1];
      dcols = hidden;
    }
    if (loss)
    {
      std::vector<float> hp(gb1);
      if (cudaMemcpyAsync(hp.data(), part, sizeof(float) * gb1,
                          cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return ASGK_ERR_CUDA;
      double t = 0;
      for (float v : hp)
        t += v;
      *loss = t;
    }
    return ASGK_OK;
  }
  int adam(float lr, cudaStream_t s)
  {
    ++step;
    float const b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float const bc1 = 1.f - std::pow(b1, float(step));
    float const bc2 = 1.f - std::pow(b2, float(step));
    for (int l = 0; l < kLayers; l++)
    {
      int64_t const nw = int64_t(dims[l]) * dims[l + 1];
      k_adam<<<grid1(nw), 256, 0, s>>>(W[l], gW[l], mW[l], vW[l], nw, lr, b1,
                                       b2, eps, bc1, bc2);
      ASGK_LAUNCHED();
      k_adam<<<grid1(dims[l + 1]), 256, 0, s>>>(b[l], gb[l], mb[l], vb[l],
                                                dims[l + 1], lr, b1, b2, eps,
                                                bc1, bc2);
      ASGK_LAUNCHED();
    }
    return sync_bf16(s);
  }
};

int mlp_precondition(asgk_mlp *mlp, asgk_plan *plan, const double *v,
                     double *z, cudaStream_t s)
{
  auto *m = reinterpret_cast<mlp_state *>(mlp);
  if (!m || !plan || plan->p.rows != m->cells || plan->p.tensor != m->ts)
    return ASGK_ERR_INVALID;
  if (int rc = m->ensure_rows(m->cells))
    return rc;
  k_pc_features<<<m->cells, 128, 0, s>>>(v, m->cells, m->ts, m->d, m->lev,
                                         m->ldx, m->X, m->scale);
  ASGK_LAUNCHED();
  if (int rc = m->forward(m->cells, s))
    return rc;
  int64_t const n = int64_t(m->cells) * m->ts;
  k_pc_output<<<grid1(n), 256, 0, s>>>(m->Y, m->cells, m->ts, m->scale, z);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

} // namespace asgk

using namespace asgk;

extern "C"
{
int asgk_mlp_create(asgk_mlp **out, int d, int n, int num_cells,
                    const int *cell_levels, int max_level, int hidden,
                    uint64_t seed)
{
  if (!out || d < 1 || d > 6 || n < 1 || num_cells < 1 || !cell_levels ||
      max_level < 1 || hidden < 16 || hidden > 4096)
    return ASGK_ERR_INVALID;
  *out   = nullptr;
  auto *m = new (std::nothrow) mlp_state();
  if (!m)
    return ASGK_ERR_ALLOC;
  int ts = 1;
  for (int i = 0; i < d; i++)
    ts *= n;
  m->d      = d;
  m->ts     = ts;
  m->in     = ts + d;
  m->ldx    = (m->in + 7) / 8 * 8;
  m->hidden = hidden;
  m->cells  = num_cells;
  int const dims[kLayers + 1] = {m->in, hidden, hidden, hidden, ts};
  std::copy(dims, dims + kLayers + 1, m->dims);
  std::mt19937_64 rng(seed);
  int rc = ASGK_OK;
  for (int l = 0; l < kLayers && !rc; l++)
  {
    int64_t const nw = int64_t(dims[l]) * dims[l + 1];
    if ((rc = m->alloc(&m->W[l], nw)) || (rc = m->alloc(&m->b[l], dims[l + 1])) ||
        (rc = m->alloc(&m->Wb[l], nw)) || (rc = m->alloc(&m->gW[l], nw)) ||
        (rc = m->alloc(&m->gb[l], dims[l + 1])) || (rc = m->alloc(&m->mW[l], nw)) ||
        (rc = m->alloc(&m->vW[l], nw)) || (rc = m->alloc(&m->mb[l], dims[l + 1])) ||
        (rc = m->alloc(&m->vb[l], dims[l + 1])))
      break;
    // uniform(-a, a), a = sqrt(6 / (fan_in + fan_out)); zero biases; the
    // last layer starts small so the untrained network is close to zero
    double const a = std::sqrt(6.0 / (dims[l] + dims[l + 1])) *
                     ((l == kLayers - 1) ? 0.1 : 1.0);
    std::uniform_real_distribution<double> U(-a, a);
    std::vector<float> hw(nw);
    for (auto &w : hw)
      w = float(U(rng));
    std::vector<float> zb(dims[l + 1], 0.f);
    if (cudaMemcpy(m->W[l], hw.data(), sizeof(float) * nw, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->b[l], zb.data(), sizeof(float) * zb.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m->mW[l], 0, sizeof(float) * nw) != cudaSuccess ||
        cudaMemset(m->vW[l], 0, sizeof(float) * nw) != cudaSuccess ||
        cudaMemset(m->mb[l], 0, sizeof(float) * dims[l + 1]) != cudaSuccess ||
        cudaMemset(m->vb[l], 0, sizeof(float) * dims[l + 1]) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
  }
  if (!rc)
  {
    std::vector<float> lev(size_t(num_cells) * d);
    for (size_t i = 0; i < lev.size(); i++)
      lev[i] = float(cell_levels[i]) / float(max_level);
    if ((rc = m->alloc(&m->lev, int64_t(lev.size()))) == ASGK_OK &&
        cudaMemcpy(m->lev, lev.data(), sizeof(float) * lev.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
  }
  if (!rc)
    rc = m->sync_bf16(nullptr);
  if (!rc && cudaDeviceSynchronize() != cudaSuccess)
    rc = ASGK_ERR_CUDA;
  if (rc)
  {
    delete m;
    return rc;
  }
  *out = reinterpret_cast<asgk_mlp *>(m);
  return ASGK_OK;
}

void asgk_mlp_destroy(asgk_mlp *mlp) { delete reinterpret_cast<mlp_state *>(mlp); }

int asgk_mlp_num_params(const asgk_mlp *mlp, int64_t *count)
{
  auto const *m = reinterpret_cast<const mlp_state *>(mlp);
  if (!m || !count)
    return ASGK_ERR_INVALID;
  int64_t c = 0;
  for (int l = 0; l < kLayers; l++)
    c += int64_t(m->dims[l]) * m->dims[l + 1] + m->dims[l + 1];
  *count = c;
  return ASGK_OK;
}

// Parameters in a flat FP32 host array: per layer W (row-major in x out), b.
int asgk_mlp_get_params(const asgk_mlp *mlp, float *params)
{
  auto const *m = reinterpret_cast<const mlp_state *>(mlp);
  if (!m || !params)
    return ASGK_ERR_INVALID;
  for (int l = 0; l < kLayers; l++)
  {
    int64_t const nw = int64_t(m->dims[l]) * m->dims[l + 1];
    ASGK_CUDA(cudaMemcpy(params, m->W[l], sizeof(float) * nw, cudaMemcpyDeviceToHost));
    params += nw;
    ASGK_CUDA(cudaMemcpy(params, m->b[l], sizeof(float) * m->dims[l + 1],
                         cudaMemcpyDeviceToHost));
    params += m->dims[l + 1];
  }
  return ASGK_OK;
}

int asgk_mlp_set_params(asgk_mlp *mlp, const float *params)
{
  auto *m = reinterpret_cast<mlp_state *>(mlp);
  if (!m || !params)
    return ASGK_ERR_INVALID;
  for (int l = 0; l < kLayers; l++)
  {
    int64_t const nw = int64_t(m->dims[l]) * m->dims[l + 1];
    ASGK_CUDA(cudaMemcpy(m->W[l], params, sizeof(float) * nw, cudaMemcpyHostToDevice));
    params += nw;
    ASGK_CUDA(cudaMemcpy(m->b[l], params, sizeof(float) * m->dims[l + 1],
                         cudaMemcpyHostToDevice));
    params += m->dims[l + 1];
  }
  if (int rc = m->sync_bf16(nullptr))
    return rc;
  ASGK_CUDA(cudaDeviceSynchronize());
  return ASGK_OK;
}

// One forward + backward on host rows (X: rows x (n^d + d), T: rows x n^d,
// both FP32): returns the loss 0.5*sum((Y-T)^2)*gscale... and the gradients
// (flat, same layout as the parameters) -- the gradient check entry point.
int asgk_mlp_forward_backward(asgk_mlp *mlp, int rows, const float *X,
                              const float *T, float *Y, float *grads,
                              double *loss)
{
  auto *m = reinterpret_cast<mlp_state *>(mlp);
  if (!m || rows < 1 || !X || !T)
    return ASGK_ERR_INVALID;
  if (int rc = m->ensure_rows(rows))
    return rc;
  std::vector<bf16> xb(size_t(rows) * m->ldx, __float2bfloat16(0.f));
  for (int r = 0; r < rows; r++)
    for (int i = 0; i < m->in; i++)
      xb[size_t(r) * m->ldx + i] = __float2bfloat16(X[size_t(r) * m->in + i]);
  ASGK_CUDA(cudaMemcpy(m->X, xb.data(), sizeof(bf16) * xb.size(), cudaMemcpyHostToDevice));
  ASGK_CUDA(cudaMemcpy(m->T, T, sizeof(float) * size_t(rows) * m->ts, cudaMemcpyHostToDevice));
  if (int rc = m->forward(rows, nullptr))
    return rc;
  double l = 0;
  if (int rc = m->backward(rows, 1.0f, &l, nullptr))
    return rc;
  ASGK_CUDA(cudaDeviceSynchronize());
  if (Y)
    ASGK_CUDA(cudaMemcpy(Y, m->Y, sizeof(float) * size_t(rows) * m->ts, cudaMemcpyDeviceToHost));
  if (grads)
    for (int li = 0; li < kLayers; li++)
    {
      int64_t const nw = int64_t(m->dims[li]) * m->dims[li + 1];
      ASGK_CUDA(cudaMemcpy(grads, m->gW[li], sizeof(float) * nw, cudaMemcpyDeviceToHost));
      grads += nw;
      ASGK_CUDA(cudaMemcpy(grads, m->gb[li], sizeof(float) * m->dims[li + 1],
                           cudaMemcpyDeviceToHost));
      grads += m->dims[li + 1];
    }
  if (loss)
    *loss = 0.5 * l;
  return ASGK_OK;
}

// Trains on (v, e) pairs given as num_samples device vectors of cells*n^d
// FP64 values each (sample-major): every (sample, cell) gives one training row
// [v_c/||v_c||, levels] -> e_c/||v_c||.  Mini-batches of `batch` rows drawn
// without replacement each epoch (seeded), Adam with learning rate lr.
int asgk_mlp_train(asgk_mlp *mlp, const double *v, const double *e,
                   int num_samples, int epochs, int batch, float lr,
                   uint64_t seed, double *final_loss, asgk_stream stream)
{
  auto *m = reinterpret_cast<mlp_state *>(mlp);
  if (!m || !v || !e || num_samples < 1 || epochs < 1 || batch < 1)
    return ASGK_ERR_INVALID;
  cudaStream_t s    = static_cast<cudaStream_t>(stream);
  int64_t const all = int64_t(num_samples) * m->cells;
  if (all > (int64_t(1) << 30))
    return ASGK_ERR_UNSUPPORTED;
  batch = int(std::min<int64_t>(batch, all));
  if (int rc = m->ensure_rows(batch))
    return rc;
  int *cell_of = nullptr, *sample_of = nullptr;
  if (cudaMalloc(&cell_of, sizeof(int) * batch) != cudaSuccess ||
      cudaMalloc(&sample_of, sizeof(int) * batch) != cudaSuccess)
  {
    cudaFree(cell_of);
    return ASGK_ERR_ALLOC;
  }
  std::vector<int64_t> order(all);
  for (int64_t i = 0; i < all; i++)
    order[i] = i;
  std::mt19937_64 rng(seed);
  std::vector<int> hc(batch), hs(batch);
  double epoch_loss = 0;
  int rc            = ASGK_OK;
  for (int ep = 0; ep < epochs && !rc; ep++)
  {
    std::shuffle(order.begin(), order.end(), rng);
    epoch_loss   = 0;
    int64_t seen = 0;
    for (int64_t b0 = 0; b0 + batch <= all && !rc; b0 += batch)
    {
      for (int i = 0; i < batch; i++)
      {
        hs[i] = int(order[b0 + i] / m->cells);
        hc[i] = int(order[b0 + i] % m->cells);
      }
      if (cudaMemcpyAsync(cell_of, hc.data(), sizeof(int) * batch,
                          cudaMemcpyHostToDevice, s) != cudaSuccess ||
          cudaMemcpyAsync(sample_of, hs.data(), sizeof(int) * batch,
                          cudaMemcpyHostToDevice, s) != cudaSuccess)
      {
        rc = ASGK_ERR_CUDA;
        break;
      }
      k_train_rows<<<batch, 128, 0, s>>>(v, e, cell_of, sample_of, batch,
                                         m->ts, m->d, int64_t(m->cells) * m->ts,
                                         m->lev, m->ldx, m->X, m->T);
      if (cudaGetLastError() != cudaSuccess)
      {
        rc = ASGK_ERR_CUDA;
        break;
      }
      count_launch();
      double l = 0;
      float const gscale = 1.0f / float(int64_t(batch) * m->ts);
      if ((rc = m->forward(batch, s)) ||
          (rc = m->backward(batch, gscale, &l, s)) || (rc = m->adam(lr, s)))
        break;
      epoch_loss += l;
      seen += int64_t(batch) * m->ts;
    }
    if (seen > 0)
      epoch_loss /= double(seen);
  }
  cudaStreamSynchronize(s);
  cudaFree(cell_of);
  cudaFree(sample_of);
  if (final_loss)
    *final_loss = epoch_loss;
  return rc;
}

// z = M(v) for a full vector of cells*n^d values (device pointers).
int asgk_mlp_apply(asgk_mlp *mlp, asgk_plan *plan, const double *v, double *z,
                   asgk_stream stream)
{
  return mlp_precondition(mlp, plan, v, z, static_cast<cudaStream_t>(stream));
}

} // extern "C"
