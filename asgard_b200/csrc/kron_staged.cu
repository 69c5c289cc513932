// Staged kronmult apply for n = 3, d = 3 and 4 (the d = 4, level 7 operator
// of the implicit-step benchmark runs here).
//
// Same operator and row ownership as kron3_rows (kron_kernels.cu); what
// differs is how data reaches the FMA pipe:
//
//   * x is first repacked (one pass, padded dimension-0 slices, every slice
//     16-byte aligned), then each pair's tensor is staged in shared memory
//     by the bulk-copy engine (cp.async.bulk, completion on an mbarrier),
//     two stages per warp, so x never passes through the load/store unit
//     and lanes read their slices with conflict-free 128-bit loads; the copy
//     of the next batch is in flight while a batch is contracted.  Every
//     wait is bounded.
//   * no per-term exchange between lanes.  A pair's tensor is held by a
//     group of three lanes; lane q holds the slice x[q, :] (dimension 0 = q,
//     3^(d-1) registers).  Dimensions 1..d-1 are contracted in registers; the
//     dimension-0 factor is applied as a column: lane q adds A0(i, q) * v to
//     its partial sums of all three output slices i.  The sum over q (and
//     over the pairs held by other lanes) is taken once per row, after the
//     pair loop, by a warp butterfly and a shared-memory sum over warps.
//     This does the same 2*d*T*3^(d+1) flops per pair as the reference's
//     kronmult, with 3^d accumulators per lane instead of a transpose of
//     every pair tensor for every term.
//
// Reference operator: kronmult::cpu_sparse, src/device/asgard_spkronmult_cpu.cpp:84-433.
#include "bulk.cuh"
#include "internal.cuh"

#include <type_traits>

namespace asgk
{
__device__ int g_device_error = 0;

namespace
{
using namespace bulk;

constexpr int ipow3s(int k) { return k == 0 ? 1 : 3 * ipow3s(k - 1); }

template<int B, int E, typename F>
__device__ __forceinline__ void sfor(F &&f)
{
  if constexpr (B < E)
  {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

template<typename TC> struct padS;
template<> struct padS<double> { static constexpr int value = 10; };
template<> struct padS<float> { static constexpr int value = 12; };

template<typename TC>
__device__ __forceinline__ void ld9(const TC *__restrict__ A, TC (&a)[9])
{
#pragma unroll
  for (int i = 0; i < 9; i++)
    a[i] = __ldg(A + i);
}

__device__ __forceinline__ void ld9p(const double *__restrict__ A, double (&a)[9])
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

__device__ __forceinline__ void ld9p(const float *__restrict__ A, float (&a)[9])
{
  const float4 *v = reinterpret_cast<const float4 *>(A);
  float4 const t0 = __ldg(v), t1 = __ldg(v + 1);
  a[0] = t0.x; a[1] = t0.y; a[2] = t0.z; a[3] = t0.w;
  a[4] = t1.x; a[5] = t1.y; a[6] = t1.z; a[7] = t1.w;
  a[8] = __ldg(A + 8);
}

// w <- (I (x) A (x) I) w along the register dimension of stride S
template<int R, int S, typename TC>
__device__ __forceinline__ void fibre3(TC (&w)[R], TC const (&a)[9])
{
#pragma unroll
  for (int b = 0; b < R; b++)
  {
    if ((b / S) % 3 == 0)
    {
      TC const w0 = w[b], w1 = w[b + S], w2 = w[b + 2 * S];
      w[b]         = fma(a[6], w2, fma(a[3], w1, a[0] * w0));
      w[b + S]     = fma(a[7], w2, fma(a[4], w1, a[1] * w0));
      w[b + 2 * S] = fma(a[8], w2, fma(a[5], w1, a[2] * w0));
    }
  }
}

__device__ __forceinline__ double2 lds_f64x2(uint32_t addr)
{
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
               : "=d"(v.x), "=d"(v.y)
               : "r"(addr));
  return v;
}

// Layout of the staged x tensors.  A tensor's three dimension-0 slices
// (3^(d-1) doubles each) are stored SP doubles apart (SP even, padded), so
// every slice starts on a 16-byte boundary and a lane reads its slice with
// 128-bit loads.  In a shared-memory stage the slot of group g starts at
// chunk (16-byte unit) slot(g): the slots are packed back to back, each
// placed at the first chunk whose residue mod 8 is RES[g].  With the three
// lanes of a group reading slices SP/2 chunks apart, these residues make the
// eight lanes of every quarter-warp of a 128-bit load hit eight distinct
// bank groups (no conflicts); they were found by exhaustive search.
template<int D, typename T> struct xlayout;
template<> struct xlayout<4, double>
{
  static constexpr int SP       = 30;  // doubles per slice (15 chunks)
  static constexpr int STAGE_CH = 496; // chunks per stage of 10 slots
  // residues {0, 3, 5, 1, 6, 2, 4, 7, 0, 3}: slot(g) = 45 g + offset(g),
  // offsets {0, 6, 11, 18, 18, 25, 30, 36, 40, 46} in six bits each
  __device__ static int slot(int g)
  {
    return 45 * g + int((0xba891e65248b180ull >> (6 * g)) & 63);
  }
};
template<> struct xlayout<4, float>
{
  static constexpr int SP       = 28;  // floats per slice (7 chunks = 15 mod 8)
  static constexpr int STAGE_CH = 256;
  // the same residues and offsets as the FP64 layout
  __device__ static int slot(int g)
  {
    return 21 * g + int((0xba891e65248b180ull >> (6 * g)) & 63);
  }
};
template<> struct xlayout<3, double>
{
  static constexpr int SP       = 10;
  static constexpr int STAGE_CH = 184;
  // residues {0, 1, 7, 2, 3, 6, 4, 5, 0, 1}: slot(g) = 15 g + offset(g),
  // offsets {0, 2, 9, 13, 15, 19, 26, 28, 32, 34}
  __device__ static int slot(int g)
  {
    return 15 * g + int((0x8a071a4cf349080ull >> (6 * g)) & 63);
  }
};
template<> struct xlayout<3, float>
{
  static constexpr int SP       = 12;  // 3 chunks: residues 0..7, 0, 1
  static constexpr int STAGE_CH = 96;
  __device__ static int slot(int g) { return 9 * g; }
};

// out <- (I (x) A (x) I) in along the register dimension of stride S
template<int R, int S, typename TC>
__device__ __forceinline__ void fibre3_from(TC const (&in)[R], TC (&out)[R],
                                            TC const (&a)[9])
{
#pragma unroll
  for (int b = 0; b < R; b++)
  {
    if ((b / S) % 3 == 0)
    {
      TC const w0 = in[b], w1 = in[b + S], w2 = in[b + 2 * S];
      out[b]         = fma(a[6], w2, fma(a[3], w1, a[0] * w0));
      out[b + S]     = fma(a[7], w2, fma(a[4], w1, a[1] * w0));
      out[b + 2 * S] = fma(a[8], w2, fma(a[5], w1, a[2] * w0));
    }
  }
}

template<int D, typename TC, int NW, int NS>
struct staged_shape
{
  using L = xlayout<D, TC>;
  static constexpr int TS    = ipow3s(D);     // tensor entries (odd)
  static constexpr int R     = ipow3s(D - 1); // registers per lane
  static constexpr int G     = 10;            // three-lane groups per warp
  static constexpr int SP    = L::SP;
  static constexpr int XP    = 3 * SP;        // elements per repacked tensor
  static constexpr int EPC   = 16 / int(sizeof(TC)); // elements per chunk
  static constexpr int NCH   = (R + EPC - 1) / EPC;  // 128-bit reads per slice
  static constexpr uint32_t COPY_BYTES = uint32_t(sizeof(TC)) * XP;
  static constexpr int STAGE_CH = L::STAGE_CH; // chunks per stage
  static_assert(SP >= NCH * EPC && (SP * sizeof(TC)) % 16 == 0, "slice padding");
  static_assert(COPY_BYTES % 16 == 0, "bulk copies move 16-byte multiples");
  static constexpr size_t bar_bytes  = size_t(NW) * NS * 8;
  static constexpr size_t red_off    = (bar_bytes + 127) / 128 * 128;
  static constexpr size_t xs_off     = (red_off + size_t(NW) * TS * sizeof(TC) + 127) / 128 * 128;
  static constexpr size_t smem_bytes = xs_off + size_t(NW) * NS * STAGE_CH * 16;
};

// x (cols tensors of 3^d doubles) -> xp (cols tensors of 3*SP values of the
// compute type, each dimension-0 slice padded to SP with zeros)
template<int D, typename T>
__global__ void k_repack_x(const double *__restrict__ x, int64_t cols,
                           T *__restrict__ xp)
{
  constexpr int R  = ipow3s(D - 1);
  constexpr int SP = xlayout<D, T>::SP;
  int64_t const total = cols * 3 * SP;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total;
       i += int64_t(gridDim.x) * blockDim.x)
  {
    int64_t const c = i / (3 * SP);
    int const r     = int(i - c * 3 * SP);
    int const q     = r / SP;
    int const m     = r - q * SP;
    xp[i]           = (m < R) ? static_cast<T>(x[c * 3 * R + q * R + m]) : T(0);
  }
}

__device__ __forceinline__ float4 lds_f32x4(uint32_t addr)
{
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(addr));
  return v;
}

// the R values of a slice at shared address a (128-bit loads)
template<int R, int NCH>
__device__ __forceinline__ void load_slice(uint32_t a, double (&w)[R])
{
#pragma unroll
  for (int j = 0; j < NCH; j++)
  {
    double2 const v = lds_f64x2(a + 16u * j);
    w[2 * j] = v.x;
    if (2 * j + 1 < R)
      w[2 * j + 1] = v.y;
  }
}
template<int R, int NCH>
__device__ __forceinline__ void load_slice(uint32_t a, float (&w)[R])
{
#pragma unroll
  for (int j = 0; j < NCH; j++)
  {
    float4 const v = lds_f32x4(a + 16u * j);
    w[4 * j] = v.x;
    if (4 * j + 1 < R) w[4 * j + 1] = v.y;
    if (4 * j + 2 < R) w[4 * j + 2] = v.z;
    if (4 * j + 3 < R) w[4 * j + 3] = v.w;
  }
}

template<int D, typename TC, index_mode MODE, bool EULER, int NW, int NS>
__global__ void __launch_bounds__(NW * 32, sizeof(TC) == 4 ? 3 : 2)
    kron3_staged(int terms, const int64_t *__restrict__ row_ptr,
                 const int *__restrict__ row_order, const int *__restrict__ col,
                 const int *__restrict__ idx, const TC *__restrict__ vF,
                 double alpha, const TC *__restrict__ xp,
                 const double *__restrict__ x, double beta,
                 double *__restrict__ y, double ex)
{
  using S = staged_shape<D, TC, NW, NS>;
  using L = typename S::L;
  constexpr int R  = S::R;
  constexpr int TS = S::TS;
  constexpr int G  = S::G;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  TC *red        = reinterpret_cast<TC *>(smem_raw + S::red_off);
  unsigned char *xs = smem_raw + S::xs_off;

  int const warp    = threadIdx.x >> 5;
  int const lane    = threadIdx.x & 31;
  int const g       = lane / 3;
  int const q       = lane - 3 * g;
  bool const laneok = g < G;
  int const gg      = laneok ? g : 0;
  uint64_t *wbar    = bars + warp * NS;
  unsigned char *wxs = xs + size_t(warp) * NS * S::STAGE_CH * 16;
  // this lane's slot and slice, as a byte offset inside a stage
  uint32_t const slot_off  = uint32_t(L::slot(gg)) * 16u;
  uint32_t const slice_off = slot_off + uint32_t(q * S::SP * sizeof(TC));
  uint32_t const wxs_u32   = smem_u32(wxs);

  int const row      = row_order[blockIdx.x];
  int64_t const pbeg = row_ptr[row];
  int64_t const pend = row_ptr[row + 1];
  int64_t const np   = pend - pbeg;
  // batches of G consecutive pairs, interleaved over the warps
  int64_t const first = int64_t(warp) * G;
  int const nb = (np > first) ? int((np - first + int64_t(NW) * G - 1) / (int64_t(NW) * G)) : 0;

  if (lane == 0)
  {
#pragma unroll
    for (int s = 0; s < NS; s++)
      mbar_init(wbar + s, 1);
    mbar_init_fence();
  }
  __syncwarp();

  auto issue = [&](int bb) {
    int const st     = bb % NS;
    int64_t const pb = pbeg + (int64_t(bb) * NW + warp) * G;
    int const nact   = (pend - pb < G) ? int(pend - pb) : G;
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0)
      mbar_arrive_expect_tx(wbar + st, uint32_t(nact) * S::COPY_BYTES);
    __syncwarp();
    if (laneok && q == 0 && g < nact)
    {
      const TC *src = xp + int64_t(__ldcs(col + pb + g)) * S::XP;
      bulk_g2s(wxs + size_t(st) * S::STAGE_CH * 16 + slot_off, src,
               S::COPY_BYTES, wbar + st);
    }
  };

  TC acc[3 * R];
#pragma unroll
  for (int e = 0; e < 3 * R; e++)
    acc[e] = TC(0);

  // FP32: a lane's slice lives in registers for all terms, so a stage is
  // refilled as soon as it has been read (NS batches ahead).  FP64 (two
  // registers per value, 3^d accumulators): the slice is re-read from the
  // stage at every term, so the refill targets the stage consumed in the
  // previous batch (NS - 1 ahead), issued before the contraction.
  constexpr bool XREG = sizeof(TC) == 4;
  constexpr int PRE   = XREG ? NS : NS - 1;
  static_assert(PRE >= 1, "at least one batch of look-ahead");
  int issued = 0;
  for (; issued < PRE && issued < nb; issued++)
    issue(issued);

  constexpr int PAD  = padS<TC>::value;
  for (int b = 0; b < nb; b++)
  {
    int const st = b % NS;
    if (!mbar_wait_bounded(wbar + st, uint32_t((b / NS) & 1)))
    {
      if (lane == 0)
        atomicExch(&g_device_error, int(ASGK_ERR_DEVICE_TIMEOUT));
      // let the copies still in flight land before the CTA's shared memory
      // is released (bounded as well), then skip the remaining pairs
      for (int bb = b; bb < issued; bb++)
        mbar_wait_bounded(wbar + bb % NS, uint32_t((bb / NS) & 1));
      break;
    }
    if constexpr (!XREG)
    {
      if (issued < nb)
      {
        issue(issued);
        issued++;
      }
    }
    int64_t const p = pbeg + (int64_t(b) * NW + warp) * G + g;
    bool const act  = laneok && p < pend;
    uint32_t const sl = wxs_u32 + uint32_t(st) * S::STAGE_CH * 16u + slice_off;
    TC xr[XREG ? R : 1];
    int cn[D];
    if (act)
    {
      if constexpr (XREG)
        load_slice<R, S::NCH>(sl, xr);
      if constexpr (MODE == index_mode::conn)
      {
#pragma unroll
        for (int k = 0; k < D; k++)
          cn[k] = __ldcs(idx + p * D + k); // streamed: keep L1 for factors
      }
    }
    if constexpr (XREG)
    {
      if (issued < nb)
      {
        issue(issued);
        issued++;
      }
    }
    if (act)
    {
#pragma unroll 1
      for (int t = 0; t < terms; t++)
      {
        TC w[R];
        if constexpr (!XREG)
          load_slice<R, S::NCH>(sl, w);
        auto blk = [&](int k) -> const TC * {
          if constexpr (MODE == index_mode::conn)
            return vF + uint32_t(((cn[k] * D + k) * terms + t) * PAD);
          else
            return vF + __ldcs(idx + (p * terms + t) * D + k);
        };
        // dimensions 1..D-1 live in registers: register m <-> (i_1 .. i_{D-1})
        // (FP32: the first one reads the slice registers, so they need no
        // copy per term)
        sfor<1, D>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          TC a[9];
          if constexpr (MODE == index_mode::conn)
            ld9p(blk(k), a);
          else
            ld9(blk(k), a);
          if constexpr (XREG && k == 1)
            fibre3_from<R, ipow3s(D - 1 - k)>(xr, w, a);
          else
            fibre3<R, ipow3s(D - 1 - k)>(w, a);
        });
        // dimension 0: this lane holds input slice q; column q of A0
        // scatters it to the three output slices
        const TC *a0 = blk(0) + 3 * q;
        TC const c0 = __ldg(a0), c1 = __ldg(a0 + 1), c2 = __ldg(a0 + 2);
#pragma unroll
        for (int m = 0; m < R; m++)
        {
          acc[m]         = fma(c0, w[m], acc[m]);
          acc[R + m]     = fma(c1, w[m], acc[R + m]);
          acc[2 * R + m] = fma(c2, w[m], acc[2 * R + m]);
        }
      }
    }
  }

  // sum the row's partial tensors over the lanes of the warp (through the
  // warp's stage buffers, idle now: all copies have landed), one output
  // slice at a time, then over the warps
  static_assert(32 * R * sizeof(TC) <= NS * S::STAGE_CH * 16, "stage buffers too small for the reduction");
  TC *wred = reinterpret_cast<TC *>(wxs);
#pragma unroll
  for (int i = 0; i < 3; i++)
  {
    __syncwarp();
#pragma unroll
    for (int m = 0; m < R; m++)
      wred[lane * R + m] = acc[i * R + m]; // odd stride: no bank conflicts
    __syncwarp();
    if (lane < R)
    {
      TC s = TC(0);
#pragma unroll 6
      for (int l = 0; l < 3 * G; l++)
        s += wred[l * R + lane];
      red[warp * TS + i * R + lane] = s;
    }
  }
  __syncthreads();
  int64_t const base = int64_t(row) * TS;
  for (int i = threadIdx.x; i < TS; i += NW * 32)
  {
    TC s = TC(0);
#pragma unroll
    for (int ww = 0; ww < NW; ww++)
      s += red[ww * TS + i];
    double v = alpha * static_cast<double>(s);
    if constexpr (EULER)
      v += ex * x[base + i];
    if (beta != 0.0)
      v += beta * y[base + i];
    y[base + i] = v;
  }
}

constexpr int kStagedWarps = 4;
// two stages per warp: shared memory is carved out of L1, which holds the
// factor blocks (about 100 KB per output cell at d = 4, level 7); FP32 stages
// are half the size and three CTAs share an SM
template<typename TC>
constexpr int kStagedStages = 2;

template<int D, typename TC, index_mode MODE, bool EULER>
int launch_staged_t(plan_data const &p, const TC *vF, double alpha,
                    const TC *xp, const double *x, double beta, double *y,
                    double ex, cudaStream_t s)
{
  using S     = staged_shape<D, TC, kStagedWarps, kStagedStages<TC>>;
  auto kern   = kron3_staged<D, TC, MODE, EULER, kStagedWarps, kStagedStages<TC>>;
  static bool configured = false;
  if (!configured)
  {
    ASGK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(S::smem_bytes)));
    configured = true;
  }
  kern<<<p.rows, kStagedWarps * 32, S::smem_bytes, s>>>(
      p.terms, p.row_ptr, p.row_order, p.col, p.idx, vF, alpha, xp, x, beta,
      y, ex);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

template<int D, typename TC>
int launch_staged_d(plan_data const &p, double alpha, const double *x,
                    double beta, double *y, double ex, cudaStream_t s)
{
  using S = staged_shape<D, TC, kStagedWarps, kStagedStages<TC>>;
  int64_t const total = int64_t(p.cols) * S::XP;
  int const blocks    = int(std::min<int64_t>((total + 255) / 256, 4096));
  TC *xp              = reinterpret_cast<TC *>(p.xs);
  k_repack_x<D, TC><<<blocks, 256, 0, s>>>(x, p.cols, xp);
  ASGK_LAUNCHED();
  const TC *vF;
  bool const conn = p.mode == index_mode::conn;
  if constexpr (std::is_same_v<TC, double>)
    vF = conn ? p.vP64 : p.vA64;
  else
    vF = conn ? p.vP32 : p.vA32;
  bool const euler = ex != 0.0;
  if (conn)
    return euler ? launch_staged_t<D, TC, index_mode::conn, true>(p, vF, alpha, xp, x, beta, y, ex, s)
                 : launch_staged_t<D, TC, index_mode::conn, false>(p, vF, alpha, xp, x, beta, y, ex, s);
  return euler ? launch_staged_t<D, TC, index_mode::expanded, true>(p, vF, alpha, xp, x, beta, y, ex, s)
               : launch_staged_t<D, TC, index_mode::expanded, false>(p, vF, alpha, xp, x, beta, y, ex, s);
}

} // namespace

int64_t staged_x_doubles(int d, int n, int cols)
{
  if (n != 3)
    return 0;
  // sized for the FP64 staging (the FP32 one is smaller)
  if (d == 4)
    return int64_t(cols) * 3 * xlayout<4, double>::SP;
  if (d == 3)
    return int64_t(cols) * 3 * xlayout<3, double>::SP;
  return 0;
}

bool staged_supported(plan_data const &p)
{
  // factor offsets of the repacked blocks are computed in 32 bits
  return p.n == 3 && (p.d == 3 || p.d == 4) && p.terms > 0 && p.xs != nullptr &&
         p.nconn * p.d * p.terms * 12 < (int64_t(1) << 31);
}

int launch_staged(plan_data const &p, int precision, double alpha,
                  const double *x, double beta, double *y, double ex,
                  cudaStream_t s)
{
  if (precision == ASGK_FP64)
    return (p.d == 3) ? launch_staged_d<3, double>(p, alpha, x, beta, y, ex, s)
                      : launch_staged_d<4, double>(p, alpha, x, beta, y, ex, s);
  if (precision == ASGK_FP32)
    return (p.d == 3) ? launch_staged_d<3, float>(p, alpha, x, beta, y, ex, s)
                      : launch_staged_d<4, float>(p, alpha, x, beta, y, ex, s);
  return ASGK_ERR_UNSUPPORTED;
}

int read_device_error(int reset, int *code)
{
  int v = 0;
  ASGK_CUDA(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int)));
  if (reset && v != 0)
  {
    int const zero = 0;
    ASGK_CUDA(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int)));
  }
  // the tensor-core kernels keep their own word
  int w = 0;
  if (int rc = tc_read_error(reset, &w))
    return rc;
  *code = (v != 0) ? v : w;
  return ASGK_OK;
}

} // namespace asgk
