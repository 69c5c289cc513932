// Learned preconditioner: a per-cell network trained and run on the GPU.
//
// Network (4 layers, width H, GELU): the cell's residual block u (scaled to
// unit norm) passes through four linear layers, every hidden layer gated
// elementwise by GELU gates computed from the cell's level multi-index
// lambda (levels / max level):
//   g_l = GELU(P_l lambda + p_l),  h_1 = g_1 * (W_1 u),
//   h_l = g_l * (W_l h_{l-1}) (l = 2, 3),  f = W_4 h_3.
// f is linear in u (nonlinear in the levels), so the preconditioner
//   z_c = ||v_c|| f(v_c / ||v_c||, lambda_c) = F(lambda_c) v_c
// is a fixed linear operator, which Krylov acceleration composes with.  A
// network nonlinear in u was tried first: it approximated (I - dt K)^{-1} v
// to 30-40% on sample vectors, yet flexible GMRES stalled with it after one
// restart cycle.  An identity skip (z = v + ...) was tried next and lost the
// stiff cells' corrections to BF16 cancellation.
//
// GEMMs run on the tensor cores in BF16 with FP32 accumulation
// (mma.sync.m16n8k16) with the gating fused into their epilogues; FP32
// master weights with Adam; MSE loss on the scaled corrections.
#include "mlp.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
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
  EPI_STORE_F32 = 0, // C = acc  (or C += acc when accumulate)
  EPI_GATE      = 1, // F = acc (f32); out = acc * G (bf16)
  EPI_GATE_BWD  = 2  // out = acc * G (bf16); F = acc * Ain (f32)
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
           int ldc, const float *__restrict__ Gin,
           const float *__restrict__ Ain, float *__restrict__ Fout,
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
        else if constexpr (EPI == EPI_GATE)
        {
          int64_t const o = int64_t(r) * ldo + c;
          Fout[o]         = v;
          out[o]          = __float2bfloat16(v * Gin[o]);
        }
        else // EPI_GATE_BWD
        {
          int64_t const o = int64_t(r) * ldo + c;
          out[o]          = __float2bfloat16(v * Gin[o]);
          Fout[o]         = v * Ain[o];
        }
      }
}

template<bool TA, bool TB, int EPI>
int gemm(int M, int N, int K, const bf16 *A, int lda, const bf16 *B, int ldb,
         float *C, int ldc, const float *Gin, const float *Ain, float *Fout,
         bf16 *out, int ldo, int accumulate, cudaStream_t s)
{
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  k_gemm<TA, TB, EPI><<<grid, 128, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc,
                                           Gin, Ain, Fout, out, ldo,
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

// Gates of one layer: Q = L P + p (rows x H), G = gelu(Q).
__global__ void k_gates(const float *__restrict__ L, int rows, int d,
                        const float *__restrict__ P,
                        const float *__restrict__ p, int H,
                        float *__restrict__ Q, float *__restrict__ G)
{
  int64_t const n = int64_t(rows) * H;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    int64_t const r = i / H;
    int const c     = int(i % H);
    float q         = p[c];
    for (int k = 0; k < d; k++)
      q += L[r * d + k] * P[k * H + c];
    Q[i] = q;
    G[i] = gelu(q);
  }
}

// Gate gradients: dq = dG * gelu'(Q); gP[k][c] = sum_r L[r][k] dq[r][c],
// gp[c] = sum_r dq[r][c].  One block per column c, the rows split over the
// block's threads and reduced in shared memory (fixed order).
__global__ void __launch_bounds__(128)
    k_gate_grad(const float *__restrict__ L, int rows, int d,
                const float *__restrict__ Q, const float *__restrict__ dG,
                int H, float *__restrict__ gP, float *__restrict__ gp)
{
  __shared__ float sh[7][128];
  int const c = blockIdx.x;
  float acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int r = threadIdx.x; r < rows; r += blockDim.x)
  {
    int64_t const i = int64_t(r) * H + c;
    float const dq  = dG[i] * dgelu(Q[i]);
    for (int k = 0; k < d; k++)
      acc[k] += L[int64_t(r) * d + k] * dq;
    acc[6] += dq;
  }
  for (int k = 0; k < 7; k++)
    sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1)
  {
    if (threadIdx.x < o)
      for (int k = 0; k < 7; k++)
        sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
  {
    for (int k = 0; k < d; k++)
      gP[k * H + c] = sh[k][0];
    gp[c] = sh[6][0];
  }
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

// Adam with decoupled weight decay on the first n_decay entries (the u-path
// weights W1..W4): the correction is pulled towards zero -- the identity
// preconditioner -- in directions the training residuals do not constrain.
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, int64_t n,
                       int64_t n_decay, float lr, float wd, float b1, float b2,
                       float eps, float bc1, float bc2)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    float const gi = g[i];
    float const mi = b1 * m[i] + (1.f - b1) * gi;
    float const vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i]           = mi;
    v[i]           = vi;
    float wi       = w[i];
    if (i < n_decay)
      wi -= lr * wd * wi;
    w[i] = wi - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// Preconditioner inputs: one row per cell, U = v_c / s_c and the level
// features, with s_c = ||v_c||_2 (1 when v_c = 0) kept for the output.
__global__ void k_pc_features(const double *__restrict__ v, int cells, int ts,
                              int d, const float *__restrict__ lev,
                              bf16 *__restrict__ U, float *__restrict__ Lr,
                              double *__restrict__ s)
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
  bf16 *row        = U + int64_t(c) * ts;
  for (int i = threadIdx.x; i < ts; i += blockDim.x)
    row[i] = __float2bfloat16(float(vc[i] / sc));
  for (int i = threadIdx.x; i < d; i += blockDim.x)
    Lr[int64_t(c) * d + i] = lev[int64_t(c) * d + i];
  if (threadIdx.x == 0)
    s[c] = (nrm > 0) ? nrm : 0.0;
}

// z_c = s_c * y_c (+ z_c when a base preconditioner's output is already in
// z).  The network predicts the correction itself, not its difference from
// v: for a stiff cell the correction is a small multiple of v_c, and forming
// it as v_c + (a BF16 quantity close to -v_c) would cancel away all of its
// digits.
__global__ void k_pc_output(const float *__restrict__ y, int cells, int ts,
                            const double *__restrict__ s,
                            const double *__restrict__ v,
                            double *__restrict__ z, int accumulate)
{
  (void)v;
  int64_t const n = int64_t(cells) * ts;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    z[i] = (accumulate ? z[i] : 0.0) + s[i / ts] * double(y[i]);
}

// Training rows from (v, e) cell pairs: U = v_c/s_c, levels, and the target
// T = e_c/s_c.
__global__ void k_train_rows(const double *__restrict__ v,
                             const double *__restrict__ e,
                             const int *__restrict__ cell_of_row,
                             const int *__restrict__ sample_of_row, int rows,
                             int ts, int d, int64_t stride,
                             const float *__restrict__ lev,
                             bf16 *__restrict__ U, float *__restrict__ Lr,
                             float *__restrict__ T)
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
    U[int64_t(r) * ts + i] = __float2bfloat16(float(v[base + i] / sc));
    T[int64_t(r) * ts + i] = float(e[base + i] / sc);
  }
  for (int i = threadIdx.x; i < d; i += blockDim.x)
    Lr[int64_t(r) * d + i] = lev[int64_t(c) * d + i];
}

int grid1(int64_t n) { return int(std::min<int64_t>(1024, (n + 255) / 256)); }

__global__ void k_sub(const double *__restrict__ a, const double *__restrict__ b,
                      double *__restrict__ c, int64_t n)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    c[i] = a[i] - b[i];
}

// partial sums of squares per block (<= 1024 blocks of 256 threads)
__global__ void k_sumsq(const double *__restrict__ x, int64_t n,
                        double *__restrict__ part)
{
  __shared__ double sh[256];
  double acc = 0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    acc += x[i] * x[i];
  sh[threadIdx.x] = acc;
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

// dY_c = coef * s_c * g_c (bf16): gradient of the residual-space loss with
// respect to the network output of cell c
__global__ void k_resid_grad(const double *__restrict__ g,
                             const double *__restrict__ sc, int cells, int ts,
                             double coef, bf16 *__restrict__ dY)
{
  int64_t const n = int64_t(cells) * ts;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    dY[i] = __float2bfloat16(float(coef * sc[i / ts] * g[i]));
}

} // namespace

// Device-resident network and its training state.  All parameters live in
// one flat FP32 buffer (layout of asgk_mlp_get_params): W1 (ts x H),
// W2 (H x H), W3 (H x H), W4 (H x ts), then for l = 1..3 the gate weights
// P_l (d x H) and biases p_l (H).
struct mlp_state
{
  int d = 0, ts = 0, hidden = 0, cells = 0;
  int64_t off_W[kLayers] = {}, off_P[3] = {}, off_p[3] = {}, nparams = 0;
  int64_t off_Wb[kLayers] = {}, nWb = 0;
  float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
  bf16 *Wb = nullptr;    // BF16 copies of W1..W4
  float *lev = nullptr;  // cells x d level features (levels / max level)
  // activations for up to cap rows
  int cap = 0;
  bf16 *U = nullptr;                 // rows x ts
  float *Lr = nullptr;               // rows x d
  float *Q[3] = {}, *G[3] = {};      // gate pre-activations and gates
  float *A[3] = {};                  // u-path pre-gate activations
  bf16 *Hh[3] = {};                  // gated activations (bf16)
  float *Y = nullptr, *T = nullptr, *part = nullptr;
  bf16 *dY = nullptr, *dA[3] = {};
  float *dG[3] = {};
  double *scale = nullptr;
  int *rows_cell = nullptr;          // identity map cell -> row for inference
  int64_t step = 0;
  float weight_decay = 0.05f;
  asgk_jacobi *base = nullptr;       // z = base(v) + network(v) when set
  std::vector<void *> owned;

  float *W(int l) { return params + off_W[l]; }
  float *gW(int l) { return grads + off_W[l]; }
  bf16 *Wbf(int l) { return Wb + off_Wb[l]; }
  int fan_in(int l) const { return l == 0 ? ts : hidden; }
  int fan_out(int l) const { return l == kLayers - 1 ? ts : hidden; }

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
    int rc;
    int64_t const rh = int64_t(rows) * hidden;
    if ((rc = alloc(&U, int64_t(rows) * ts)) || (rc = alloc(&Lr, int64_t(rows) * d)) ||
        (rc = alloc(&Y, int64_t(rows) * ts)) || (rc = alloc(&T, int64_t(rows) * ts)) ||
        (rc = alloc(&dY, int64_t(rows) * ts)) || (rc = alloc(&part, 1024)) ||
        (rc = alloc(&scale, rows)) || (rc = alloc(&rows_cell, rows)))
      return rc;
    for (int l = 0; l < 3; l++)
      if ((rc = alloc(&Q[l], rh)) || (rc = alloc(&G[l], rh)) || (rc = alloc(&A[l], rh)) ||
          (rc = alloc(&Hh[l], rh)) || (rc = alloc(&dA[l], rh)) || (rc = alloc(&dG[l], rh)))
        return rc;
    cap = rows;
    return ASGK_OK;
  }
  int sync_bf16(cudaStream_t s)
  {
    for (int l = 0; l < kLayers; l++)
    {
      int64_t const n = int64_t(fan_in(l)) * fan_out(l);
      k_f32_to_bf16<<<grid1(n), 256, 0, s>>>(W(l), Wbf(l), n);
      ASGK_LAUNCHED();
    }
    return ASGK_OK;
  }
  // forward on rows [0, rows) of U / Lr
  int forward(int rows, cudaStream_t s)
  {
    for (int l = 0; l < 3; l++)
    {
      k_gates<<<grid1(int64_t(rows) * hidden), 256, 0, s>>>(
          Lr, rows, d, params + off_P[l], params + off_p[l], hidden, Q[l], G[l]);
      ASGK_LAUNCHED();
    }
    const bf16 *in = U;
    int in_ld      = ts;
    for (int l = 0; l < 3; l++)
    {
      if (int rc = gemm<false, false, EPI_GATE>(rows, hidden, fan_in(l), in,
                                                in_ld, Wbf(l), hidden, nullptr,
                                                0, G[l], nullptr, A[l], Hh[l],
                                                hidden, 0, s))
        return rc;
      in    = Hh[l];
      in_ld = hidden;
    }
    return gemm<false, false, EPI_STORE_F32>(rows, ts, hidden, in, hidden,
                                             Wbf(3), ts, Y, ts, nullptr,
                                             nullptr, nullptr, nullptr, 0, 0, s);
  }
  // gradients of 0.5 * gscale * sum((Y - T)^2)
  int backward(int rows, float gscale, double *loss, cudaStream_t s)
  {
    int64_t const n = int64_t(rows) * ts;
    int const gb1   = grid1(n);
    k_mse_grad<<<gb1, 256, 0, s>>>(Y, T, n, gscale, dY, part);
    ASGK_LAUNCHED();
    if (int rc = backward_from_dY(rows, s))
      return rc;
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
  // parameter gradients for the output gradient already in dY
  int backward_from_dY(int rows, cudaStream_t s)
  {
    const bf16 *dcur = dY;
    int dcols        = ts;
    for (int l = kLayers - 1; l >= 0; l--)
    {
      const bf16 *act  = (l == 0) ? U : Hh[l - 1];
      int const act_ld = (l == 0) ? ts : hidden;
      if (int rc = gemm<true, false, EPI_STORE_F32>(
              fan_in(l), dcols, rows, act, act_ld, dcur, dcols, gW(l), dcols,
              nullptr, nullptr, nullptr, nullptr, 0, 0, s))
        return rc;
      if (l == 0)
        break;
      // dh = dcur W_l^T; dA = dh * G, dG = dh * A for the gated layer l-1
      if (int rc = gemm<false, true, EPI_GATE_BWD>(
              rows, hidden, dcols, dcur, dcols, Wbf(l), dcols, nullptr, 0,
              G[l - 1], A[l - 1], dG[l - 1], dA[l - 1], hidden, 0, s))
        return rc;
      dcur  = dA[l - 1];
      dcols = hidden;
    }
    for (int l = 0; l < 3; l++)
    {
      k_gate_grad<<<hidden, 128, 0, s>>>(
          Lr, rows, d, Q[l], dG[l], hidden, grads + off_P[l], grads + off_p[l]);
      ASGK_LAUNCHED();
    }
    return ASGK_OK;
  }
  int adam(float lr, cudaStream_t s)
  {
    ++step;
    float const b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float const bc1 = 1.f - std::pow(b1, float(step));
    float const bc2 = 1.f - std::pow(b2, float(step));
    k_adam<<<grid1(nparams), 256, 0, s>>>(params, grads, m1, m2, nparams,
                                          nWb, lr, weight_decay, b1, b2, eps,
                                          bc1, bc2);
    ASGK_LAUNCHED();
    return sync_bf16(s);
  }
};

int mlp_check_shape(const asgk_mlp *mlp, int rows, int tensor)
{
  auto const *m = reinterpret_cast<const mlp_state *>(mlp);
  return (m && m->cells == rows && m->ts == tensor) ? ASGK_OK : ASGK_ERR_INVALID;
}

int mlp_precondition(asgk_mlp *mlp, asgk_plan *plan, const double *v,
                     double *z, cudaStream_t s, bool low)
{
  auto *m = reinterpret_cast<mlp_state *>(mlp);
  if (!m || !plan || plan->p.rows != m->cells || plan->p.tensor != m->ts)
    return ASGK_ERR_INVALID;
  if (int rc = m->ensure_rows(m->cells))
    return rc;
  if (m->base)
    if (int rc = jacobi_apply_handle(m->base, low, const_cast<double *>(v), z,
                                     nullptr, nullptr, s)) // v only read
      return rc;
  k_pc_features<<<m->cells, 128, 0, s>>>(v, m->cells, m->ts, m->d, m->lev,
                                         m->U, m->Lr, m->scale);
  ASGK_LAUNCHED();
  if (int rc = m->forward(m->cells, s))
    return rc;
  int64_t const n = int64_t(m->cells) * m->ts;
  k_pc_output<<<grid1(n), 256, 0, s>>>(m->Y, m->cells, m->ts, m->scale, v, z,
                                       m->base != nullptr);
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
  try
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
    m->hidden = hidden;
    m->cells  = num_cells;
    int64_t o = 0, ob = 0;
    for (int l = 0; l < kLayers; l++)
    {
      m->off_W[l]  = o;
      m->off_Wb[l] = ob;
      int64_t const nw = int64_t(m->fan_in(l)) * m->fan_out(l);
      o += nw;
      ob += nw;
    }
    for (int l = 0; l < 3; l++)
    {
      m->off_P[l] = o;
      o += int64_t(d) * hidden;
      m->off_p[l] = o;
      o += hidden;
    }
    m->nparams = o;
    m->nWb     = ob;
    int rc     = ASGK_OK;
    if ((rc = m->alloc(&m->params, o)) || (rc = m->alloc(&m->grads, o)) ||
        (rc = m->alloc(&m->m1, o)) || (rc = m->alloc(&m->m2, o)) ||
        (rc = m->alloc(&m->Wb, ob)) || (rc = m->alloc(&m->lev, int64_t(num_cells) * d)))
    {
      delete m;
      return rc;
    }
    // W_l uniform(-a, a), a = sqrt(6 / (fan_in + fan_out)), the last layer
    // scaled by 0.1 (the untrained network is close to the identity map);
    // gate weights P_l uniform(-1, 1), gate biases 1 (gates start near 0.84)
    std::mt19937_64 rng(seed);
    std::vector<float> h(o, 0.f);
    for (int l = 0; l < kLayers; l++)
    {
      double const a = std::sqrt(6.0 / (m->fan_in(l) + m->fan_out(l))) *
                       ((l == kLayers - 1) ? 0.1 : 1.0);
      std::uniform_real_distribution<double> U(-a, a);
      int64_t const nw = int64_t(m->fan_in(l)) * m->fan_out(l);
      for (int64_t i = 0; i < nw; i++)
        h[m->off_W[l] + i] = float(U(rng));
    }
    std::uniform_real_distribution<double> Ug(-1.0, 1.0);
    for (int l = 0; l < 3; l++)
    {
      for (int64_t i = 0; i < int64_t(d) * hidden; i++)
        h[m->off_P[l] + i] = float(Ug(rng));
      for (int i = 0; i < hidden; i++)
        h[m->off_p[l] + i] = 1.0f;
    }
    std::vector<float> lev(size_t(num_cells) * d);
    for (size_t i = 0; i < lev.size(); i++)
      lev[i] = float(cell_levels[i]) / float(max_level);
    if (cudaMemcpy(m->params, h.data(), sizeof(float) * o, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m->m1, 0, sizeof(float) * o) != cudaSuccess ||
        cudaMemset(m->m2, 0, sizeof(float) * o) != cudaSuccess ||
        cudaMemset(m->grads, 0, sizeof(float) * o) != cudaSuccess ||
        cudaMemcpy(m->lev, lev.data(), sizeof(float) * lev.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      rc = ASGK_ERR_CUDA;
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
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

void asgk_mlp_destroy(asgk_mlp *mlp) { delete reinterpret_cast<mlp_state *>(mlp); }

int asgk_mlp_num_params(const asgk_mlp *mlp, int64_t *count)
{
  try
  {
    auto const *m = reinterpret_cast<const mlp_state *>(mlp);
    if (!m || !count)
      return ASGK_ERR_INVALID;
    *count = m->nparams;
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

int asgk_mlp_get_params(const asgk_mlp *mlp, float *params)
{
  try
  {
    auto const *m = reinterpret_cast<const mlp_state *>(mlp);
    if (!m || !params)
      return ASGK_ERR_INVALID;
    ASGK_CUDA(cudaMemcpy(params, m->params, sizeof(float) * m->nparams,
                         cudaMemcpyDeviceToHost));
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

int asgk_mlp_set_params(asgk_mlp *mlp, const float *params)
{
  try
  {
    auto *m = reinterpret_cast<mlp_state *>(mlp);
    if (!m || !params)
      return ASGK_ERR_INVALID;
    ASGK_CUDA(cudaMemcpy(m->params, params, sizeof(float) * m->nparams,
                         cudaMemcpyHostToDevice));
    if (int rc = m->sync_bf16(nullptr))
      return rc;
    ASGK_CUDA(cudaDeviceSynchronize());
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

// One forward + backward pass on host rows (X: rows x (n^d + d) = residual
// block then level features, T: rows x n^d, FP32): Y, loss = 0.5*sum((Y-T)^2)
// and the gradients in the parameter layout -- the gradient-check entry.
int asgk_mlp_forward_backward(asgk_mlp *mlp, int rows, const float *X,
                              const float *T, float *Y, float *grads,
                              double *loss)
{
  try
  {
    auto *m = reinterpret_cast<mlp_state *>(mlp);
    if (!m || rows < 1 || !X || !T)
      return ASGK_ERR_INVALID;
    if (int rc = m->ensure_rows(rows))
      return rc;
    int const in = m->ts + m->d;
    std::vector<bf16> u(size_t(rows) * m->ts);
    std::vector<float> lr(size_t(rows) * m->d);
    for (int r = 0; r < rows; r++)
    {
      for (int i = 0; i < m->ts; i++)
        u[size_t(r) * m->ts + i] = __float2bfloat16(X[size_t(r) * in + i]);
      for (int i = 0; i < m->d; i++)
        lr[size_t(r) * m->d + i] = X[size_t(r) * in + m->ts + i];
    }
    ASGK_CUDA(cudaMemcpy(m->U, u.data(), sizeof(bf16) * u.size(), cudaMemcpyHostToDevice));
    ASGK_CUDA(cudaMemcpy(m->Lr, lr.data(), sizeof(float) * lr.size(), cudaMemcpyHostToDevice));
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
      ASGK_CUDA(cudaMemcpy(grads, m->grads, sizeof(float) * m->nparams, cudaMemcpyDeviceToHost));
    if (loss)
      *loss = 0.5 * l;
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

// Trains on (v, e) pairs given as num_samples device vectors of cells*n^d
// FP64 values each (sample-major): every (sample, cell) gives one training row
// (v_c/||v_c||, levels) -> e_c/||v_c||.  Mini-batches of `batch` rows
// drawn without replacement each epoch (seeded), Adam with learning rate lr.
int asgk_mlp_train(asgk_mlp *mlp, const double *v, const double *e,
                   int num_samples, int epochs, int batch, float lr,
                   uint64_t seed, double *final_loss, asgk_stream stream)
{
  try
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
                                           m->lev, m->U, m->Lr, m->T);
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
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

// Residual-space training on (residual, GMRES-correction) pairs (r_k, e_k)
// with A e_k = r_k, A = I - dt K: per sample the loss is
//   ||A (M r_k - e_k)||^2 / ||r_k||^2  =  ||A M r_k - r_k||^2 / ||r_k||^2,
// the preconditioned residual, so errors along stiff directions count with
// the weight A gives them.  Its gradient needs A^T: plan_T is K^T on the same
// pair list.  One Adam step per sample (all cells of it in one batch).
int asgk_mlp_train_residual(asgk_mlp *mlp, asgk_plan *plan, asgk_plan *plan_T,
                            double dt, const double *r, const double *e,
                            int num_samples, int epochs, float lr,
                            int precision, uint64_t seed, double *final_loss,
                            asgk_stream stream)
{
  try
  {
    auto *m = reinterpret_cast<mlp_state *>(mlp);
    if (!m || !plan || !plan_T || !r || !e || num_samples < 1 || epochs < 1)
      return ASGK_ERR_INVALID;
    if (plan->p.rows != m->cells || plan->p.tensor != m->ts ||
        plan_T->p.rows != m->cells || plan_T->p.tensor != m->ts)
      return ASGK_ERR_INVALID;
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    int64_t const N = int64_t(m->cells) * m->ts;
    if (int rc = m->ensure_rows(m->cells))
      return rc;
    double *buf = nullptr, *part = nullptr;
    if (cudaMalloc(&buf, sizeof(double) * 4 * N) != cudaSuccess ||
        cudaMalloc(&part, sizeof(double) * 1024) != cudaSuccess)
    {
      cudaGetLastError();
      cudaFree(buf);
      return ASGK_ERR_ALLOC;
    }
    double *z = buf, *dv = buf + N, *q = buf + 2 * N, *g = buf + 3 * N;
    int const gb = grid1(N);
    std::vector<double> hp(gb);
    auto sumsq = [&](const double *x, double &out) -> int {
      k_sumsq<<<gb, 256, 0, s>>>(x, N, part);
      ASGK_LAUNCHED();
      ASGK_CUDA(cudaMemcpyAsync(hp.data(), part, sizeof(double) * gb,
                                cudaMemcpyDeviceToHost, s));
      ASGK_CUDA(cudaStreamSynchronize(s));
      out = 0;
      for (double v : hp)
        out += v;
      return ASGK_OK;
    };
    std::vector<int> order(num_samples);
    for (int i = 0; i < num_samples; i++)
      order[i] = i;
    std::mt19937_64 rng(seed);
    double epoch_loss = 0;
    int rc            = ASGK_OK;
    for (int ep = 0; ep < epochs && !rc; ep++)
    {
      std::shuffle(order.begin(), order.end(), rng);
      epoch_loss = 0;
      for (int it = 0; it < num_samples && !rc; it++)
      {
        const double *rk = r + int64_t(order[it]) * N;
        const double *ek = e + int64_t(order[it]) * N;
        double nr2 = 0, nq2 = 0;
        if ((rc = sumsq(rk, nr2)))
          break;
        if (!(nr2 > 0))
          continue;
        k_pc_features<<<m->cells, 128, 0, s>>>(rk, m->cells, m->ts, m->d, m->lev,
                                               m->U, m->Lr, m->scale);
        if (cudaGetLastError() != cudaSuccess)
        {
          rc = ASGK_ERR_CUDA;
          break;
        }
        count_launch();
        if ((rc = m->forward(m->cells, s)))
          break;
        k_pc_output<<<gb, 256, 0, s>>>(m->Y, m->cells, m->ts, m->scale, rk, z, 0);
        k_sub<<<gb, 256, 0, s>>>(z, ek, dv, N);
        if (cudaGetLastError() != cudaSuccess)
        {
          rc = ASGK_ERR_CUDA;
          break;
        }
        count_launch(2);
        if ((rc = asgk_apply_euler(plan, precision, dt, 1.0, dv, 0.0, q, stream)) ||
            (rc = sumsq(q, nq2)) ||
            (rc = asgk_apply_euler(plan_T, precision, dt, 1.0, q, 0.0, g, stream)))
          break;
        epoch_loss += nq2 / nr2;
        k_resid_grad<<<gb, 256, 0, s>>>(g, m->scale, m->cells, m->ts, 2.0 / nr2,
                                        m->dY);
        if (cudaGetLastError() != cudaSuccess)
        {
          rc = ASGK_ERR_CUDA;
          break;
        }
        count_launch();
        if ((rc = m->backward_from_dY(m->cells, s)) || (rc = m->adam(lr, s)))
          break;
      }
      epoch_loss /= num_samples;
    }
    cudaStreamSynchronize(s);
    cudaFree(buf);
    cudaFree(part);
    if (final_loss)
      *final_loss = epoch_loss;
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

int asgk_mlp_set_base(asgk_mlp *mlp, asgk_jacobi *base)
{
  try
  {
    auto *m = reinterpret_cast<mlp_state *>(mlp);
    if (!m)
      return ASGK_ERR_INVALID;
    // the base is applied to the network's full vectors (cells * n^d)
    if (base != nullptr && jacobi_check_shape(base, m->cells, m->ts))
      return ASGK_ERR_INVALID;
    m->base = base;
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

// z = M(v) for a full vector of cells*n^d values (device pointers).
int asgk_mlp_apply(asgk_mlp *mlp, asgk_plan *plan, const double *v, double *z,
                   asgk_stream stream)
{
  try
  {
    return mlp_precondition(mlp, plan, v, z, static_cast<cudaStream_t>(stream),
                            false);
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
