// Tensor-core form of the global Kronecker operator (precision ASGK_BF16):
// BF16 operands on the fifth-generation tensor cores (tcgen05.mma,
// kind::f16) with FP32 accumulators in tensor memory, used as the inner
// operator of the mixed-precision solves (FP64 refinement around it).  No
// counterpart in the reference, whose kronmult runs FP64/FP32 on CUDA cores
// (src/device/asgard_spkronmult_cycle2.hpp:17-382, global form
// src/device/asgard_glkronmult_cpu.cpp:103-181).
//
// The plan's terms act in one dimension each, so K = sum_k K_k and K_k
// couples only the cells of a pencil along k (cells that agree outside k).
// On a pencil P of p cells K_k is A_P (x) I, A_P (3p x 3p) the 1D operator of
// dimension k restricted to the pencil's 1D cells: one matrix per distinct
// 1D cell set (on a standard sparse grid one per pencil size).  Stacking the
// pencils of one such class, the product is a GEMM:
//   Y[(P, f), n] = sum_kk X[(P, f), kk] A_P[n, kk],
// rows (pencil, fibre f: the 3^(d-1) index combinations of the other
// dimensions), kk = (cell i of P, polynomial c along k), n = (cell i', c').
// A tile is 128 rows (M = 128, one TMEM lane each; a CTA takes one tile, or
// four of one class for pencils of up to 8 cells): its threads gather the
// rows' X into shared memory as BF16 in the no-swizzle K-major layout, the
// class matrix arrives in 64-column chunks by bulk copy (laid out on the
// host in the same layout), and one thread issues the MMAs (K = 16 each; N
// <= 256 per instruction, two halves above) into TMEM; chunks are
// double-buffered, their reuse ordered by tcgen05.commit on mbarriers.  The
// epilogue reads the accumulators (tcgen05.ld, each warp its 32 lanes) and
// adds them into the cells' values.  Every cell lies in exactly one pencil
// per dimension, so the launches of one dimension (one per TMEM size) write
// disjoint values and run concurrently on side streams; matrices of 3 x 32
// cells and more take 512-thread CTAs whose four thread groups split each
// tile's gather and epilogue; dimensions follow one another through an FP32
// sum vector and the last one forms
//   y = beta y + alpha (sum_k K_k x + n_identity x) + ex x
// in FP64.  x is rounded to BF16 once per apply (a conversion pass); the
// same summation order every call, so results are bit-reproducible.
#include "bulk.cuh"
#include "internal.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <vector>

namespace asgk
{
// set by a bounded wait of the tensor-core kernel that gave up
__device__ int g_tc_error = 0;

namespace
{
using namespace bulk;

constexpr int kTcRows    = 128; // rows per tile: M of the MMA, TMEM lanes
constexpr int kTcK       = 64;  // K columns per staged chunk (four MMAs)
constexpr int kTcThreads = 128;     // small matrices (up to 64 TMEM columns)
constexpr int kTcThreadsWide = 512; // matrices of 3 x 32 cells and more
constexpr int kTcTilesSmall  = 4;   // tiles per CTA for matrices of up to 3 x 8 cells

constexpr int ipow3t(int k) { return k <= 0 ? 1 : 3 * ipow3t(k - 1); }

// ---- tcgen05 / TMEM primitives (inline PTX, sm_100a) ----------------------

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(cols)
               : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the two 8x16-byte core matrices of a K = 16 step), stride
// byte offset (between 8-row groups), descriptor version 1 at bit 46.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return uint64_t((addr >> 4) & 0x3fff) | (uint64_t((lbo >> 4) & 0x3fff) << 16) |
         (uint64_t((sbo >> 4) & 0x3fff) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1),
// A and B BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) |
         (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
               : "memory");
}

// arrives on bar once every MMA this thread issued before has completed
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 16 consecutive FP32 columns of the calling thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
               "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

} // namespace

// One class of pencils of one dimension: the class matrix (R = 3p rows and
// columns, padded to Np x Kp) and the pencils that use it.
struct tc_group
{
  int R, Np, Kp, img_off; // img_off: first BF16 element of its chunk images
  int pen0, npen;         // its pencils in pen_start
  int pad0, pad1;
};

// one launch: the tiles of one dimension whose matrices need `cols` TMEM
// columns (a power of two >= Np)
struct tc_launch
{
  int k = 0, cols = 0, ntiles = 0, np_max = 0, kp_max = 0, nt = 0, tpc = 1;
  int abytes = 0, bbytes = 0, nbuf = 0; // chunk buffers sized for this launch
  size_t smem       = 0;
  int2 *tiles       = nullptr; // (group, first row)
};

struct tc_class_host
{
  int k = 0;             // a dimension whose operator the class matrix holds
  std::vector<int> set;  // the pencil's 1D cells along k, ascending
  int R = 0, Np = 0, Kp = 0, img_off = 0;
};

struct tc_data
{
  int d = 0, rows = 0, ts = 0;
  std::vector<int> dims; // dimensions with terms, ascending
  std::vector<tc_launch> launches;
  std::vector<tc_class_host> classes;
  int64_t img_len       = 0;
  tc_group *groups      = nullptr;
  int *pen_start        = nullptr; // [pencils + 1] offsets into pen_cells
  int *pen_cells        = nullptr;
  __nv_bfloat16 *img    = nullptr; // class matrices, chunked, K-major core-matrix layout
  __nv_bfloat16 *xb     = nullptr; // x rounded to BF16
  float *acc            = nullptr; // FP32 sum over the dimensions
  int64_t bytes         = 0;
  // the launches of one dimension touch disjoint cells and run concurrently:
  // the first on the caller's stream, the others on side streams forked and
  // joined by events (parallel branches when recorded into a graph)
  std::vector<cudaStream_t> side;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  ~tc_data()
  {
    for (auto st : side)
      cudaStreamDestroy(st);
    for (auto ev : join)
      cudaEventDestroy(ev);
    if (fork)
      cudaEventDestroy(fork);
    for (auto &l : launches)
      cudaFree(l.tiles);
    cudaFree(groups);
    cudaFree(pen_start);
    cudaFree(pen_cells);
    cudaFree(img);
    cudaFree(xb);
    cudaFree(acc);
  }
};

namespace
{
__global__ void k_to_bf16(const double *__restrict__ x, __nv_bfloat16 *__restrict__ xb,
                          int64_t n, const double *gate)
{
  if (gate_closed(gate))
    return;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    xb[i] = __double2bfloat16(x[i]);
}

// mode 0: acc = K_k x (first dimension); 1: acc += K_k x; 2 (last): y = beta
// y + alpha (acc + K_k x) + ex x; 3 (the only dimension): y = beta y + alpha
// K_k x + ex x.  post = 3^(D-1-k): fibre f of dimension k holds the values
// (f / post) * 3 post + c post + f % post, c = 0, 1, 2.  A CTA takes TILES
// consecutive tiles of 128 rows of one class (its MMAs share the class
// matrix; tile i accumulates in TMEM columns i * Np on), and NT / (128 TILES)
// thread groups share each row: thread t owns row t % (128 TILES) (the TMEM
// lane of its warp's lane quarter in tile (t % (128 TILES)) / 128) and group
// t / (128 TILES) takes every NP-th 8-column piece of the gather and
// 16-column piece of the epilogue.  Large pencils: one tile, four groups
// (their long chains split); pencils of 1-8 cells: four tiles, one group
// (the per-CTA set-up, matrix copy and MMA round trip shared).
template<int D, int NT, int TILES>
__global__ void __launch_bounds__(NT)
    k_tc_pencil(const int2 *__restrict__ tiles, const tc_group *__restrict__ groups,
                const int *__restrict__ pen_start, const int *__restrict__ pen_cells,
                const __nv_bfloat16 *__restrict__ img, const __nv_bfloat16 *__restrict__ xb,
                float *__restrict__ acc, int post, uint32_t cols, int abytes, int bbytes,
                int nbuf, int mode,
                double alpha, const double *__restrict__ x, double beta,
                double *__restrict__ y, double ex, const double *gate)
{
  constexpr int T = ipow3t(D), F = T / 3;
  constexpr int ROWS = kTcRows * TILES;
  constexpr int NP   = NT / ROWS;
  static_assert(NP >= 1 && NT % ROWS == 0, "thread groups");
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bbar[2], mbar[2];
  __shared__ uint32_t tslot;
  __shared__ int s_abort;
  if (gate_closed(gate))
    return;
  int const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int const row = tid % ROWS, part = tid / ROWS;
  int const ti  = row / kTcRows, r128 = row % kTcRows; // tile, lane
  int2 const tile  = tiles[blockIdx.x];
  tc_group const g = groups[tile.x];
  int const nch    = (g.Kp + kTcK - 1) / kTcK;
  unsigned char *const Abuf = smem;
  unsigned char *const Bbuf = smem + nbuf * abytes;

  if (tid == 0)
  {
    mbar_init(&bbar[0], 1);
    mbar_init(&bbar[1], 1);
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
    s_abort = 0;
  }
  if (warp == 0)
  {
    tmem_alloc(&tslot, cols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  uint32_t const tmem = tslot;

  // this thread's row: pencil P of the class, fibre f
  int const rowg   = tile.y + row;
  bool const valid = rowg < g.npen * F;
  int const P      = valid ? rowg / F : 0;
  int const f      = valid ? rowg - P * F : 0;
  const int *cells = pen_cells + pen_start[g.pen0 + P];
  int const base   = (f / post) * 3 * post + (f % post);

  int nh = g.Np > 256 ? 2 : 1;
  int const Nh = g.Np / nh;
  uint32_t const idesc = idesc_bf16(kTcRows, Nh);
  int committed = -1; // last chunk whose MMAs were committed
  int pending   = -1; // a chunk whose bulk copy was not seen to land
  for (int j = 0; j < nch; j++)
  {
    int const b   = j & 1;
    int const kk0 = j * kTcK;
    int const kc  = min(kTcK, g.Kp - kk0);
    // the buffers of chunk j - 2 are free once its MMAs completed
    if (j >= 2 && !mbar_wait_bounded(&mbar[b], uint32_t(((j - 2) >> 1) & 1)))
      if (lane == 0)
        s_abort = 1;
    __syncthreads();
    if (s_abort)
      break;
    unsigned char *const A = Abuf + b * abytes;
    unsigned char *const B = Bbuf + b * bbytes;
    if (tid == 0)
    {
      uint32_t const nbytes = uint32_t(g.Np) * uint32_t(kc) * 2u;
      mbar_arrive_expect_tx(&bbar[b], nbytes);
      bulk_g2s(B, img + g.img_off + int64_t(g.Np) * kk0, nbytes, &bbar[b]);
    }
    // gather the rows' chunk of X: core matrix (row / 8, column / 8) at
    // (row / 8) * kc * 16 + (column / 8) * 128 bytes, 16 bytes per row
    int const tbytes = kTcRows * kc * 2; // one tile's rows of the chunk
    unsigned char *const arow =
        A + ti * tbytes + (r128 >> 3) * (kc * 16) + (r128 & 7) * 16;
    // columns of this chunk that hold values of this row (the rest is the
    // zero padding up to Kp): pieces past them are stored as zeros without
    // loads; (cell, polynomial) of a column advance without divisions
    int const kvalid = valid ? min(kc, g.R - kk0) : 0;
    for (int e8 = part; e8 < kc / 8; e8 += NP)
    {
      unsigned short v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (e8 * 8 < kvalid)
      {
        int const kk = kk0 + e8 * 8;
        int i        = kk / 3;
        int c        = kk - 3 * i;
        int64_t off  = int64_t(cells[i]) * T + base;
#pragma unroll
        for (int q = 0; q < 8; q++)
        {
          if (e8 * 8 + q < kvalid)
            v[q] = __bfloat16_as_ushort(xb[off + c * post]);
          if (++c == 3 && q < 7)
          {
            c = 0;
            ++i;
            if (kk + q + 1 < g.R)
              off = int64_t(cells[i]) * T + base;
          }
        }
      }
      uint4 pk;
      pk.x = uint32_t(v[0]) | (uint32_t(v[1]) << 16);
      pk.y = uint32_t(v[2]) | (uint32_t(v[3]) << 16);
      pk.z = uint32_t(v[4]) | (uint32_t(v[5]) << 16);
      pk.w = uint32_t(v[6]) | (uint32_t(v[7]) << 16);
      *reinterpret_cast<uint4 *>(arow + e8 * 128) = pk;
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (warp == 0)
    {
      bool const ok = mbar_wait_bounded(&bbar[b], uint32_t((j >> 1) & 1));
      if (!ok)
      {
        pending = j;
        if (lane == 0)
          s_abort = 1;
      }
      else if (lane == 0)
      {
        tc_fence_after();
        uint32_t const a0 = smem_u32(A), b0 = smem_u32(B);
        uint32_t const sbo = uint32_t(kc) * 16u;
        for (int s = 0; s < kc / 16; s++)
          for (int t2 = 0; t2 < TILES; t2++)
          {
            uint64_t const ad =
                smem_desc(a0 + t2 * kTcRows * kc * 2 + s * 256, 128, sbo);
            for (int h = 0; h < nh; h++)
            {
              uint64_t const bd = smem_desc(b0 + h * (Nh / 8) * sbo + s * 256, 128, sbo);
              mma_bf16(tmem + uint32_t(t2 * g.Np + h * Nh), ad, bd, idesc,
                       (j > 0 || s > 0) ? 1u : 0u);
            }
          }
        mma_commit(&mbar[b]);
      }
    }
    __syncthreads();
    if (s_abort)
      break;
    committed = j;
  }
  bool done = false;
  if (committed >= 0)
    done = mbar_wait_bounded(&mbar[committed & 1], uint32_t((committed >> 1) & 1));
  if (!done || s_abort)
  {
    if (lane == 0)
      atomicExch(&g_tc_error, int(ASGK_ERR_DEVICE_TIMEOUT));
    // a copy still in flight lands before shared memory is released (bounded)
    if (warp == 0 && pending >= 0)
      mbar_wait_bounded(&bbar[pending & 1], uint32_t((pending >> 1) & 1));
  }
  tc_fence_after();
  if (done && !s_abort)
  {
    uint32_t const lanebase =
        tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(ti * g.Np);
    for (int n0 = 16 * part; n0 < g.R; n0 += 16 * NP)
    {
      uint32_t r[16];
      tmem_ld16(lanebase + uint32_t(n0), r);
      if (!valid)
        continue;
#pragma unroll
      for (int q = 0; q < 16; q++)
      {
        int const n = n0 + q;
        if (n >= g.R)
          break;
        int const i = n / 3, c = n - 3 * i;
        int64_t const idx = int64_t(cells[i]) * T + base + c * post;
        float const v     = __uint_as_float(r[q]);
        if (mode == 0)
          acc[idx] = v;
        else if (mode == 1)
          acc[idx] += v;
        else
        {
          double const kx = (mode == 2) ? double(acc[idx] + v) : double(v);
          double const yo = (beta == 0.0) ? 0.0 : beta * y[idx];
          y[idx]          = yo + alpha * kx + ex * x[idx];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
  {
    tc_fence_after();
    tmem_dealloc(tmem, cols);
  }
}

template<int D>
void *tc_kernel(int nt, int tiles)
{
  if (tiles == kTcTilesSmall)
    return reinterpret_cast<void *>(&k_tc_pencil<D, kTcThreadsWide, kTcTilesSmall>);
  return nt == kTcThreadsWide ? reinterpret_cast<void *>(&k_tc_pencil<D, kTcThreadsWide, 1>)
                              : reinterpret_cast<void *>(&k_tc_pencil<D, kTcThreads, 1>);
}

void *tc_kernel_d(int d, int nt, int tiles)
{
  switch (d)
  {
  case 1: return tc_kernel<1>(nt, tiles);
  case 2: return tc_kernel<2>(nt, tiles);
  case 3: return tc_kernel<3>(nt, tiles);
  case 4: return tc_kernel<4>(nt, tiles);
  case 5: return tc_kernel<5>(nt, tiles);
  case 6: return tc_kernel<6>(nt, tiles);
  default: return nullptr;
  }
}

template<typename T>
int upload_tc(T **dst, std::vector<T> const &src, int64_t &bytes)
{
  size_t const n = std::max<size_t>(src.size(), 1);
  ASGK_CUDA(cudaMalloc(dst, sizeof(T) * n));
  if (!src.empty())
    ASGK_CUDA(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
  bytes += int64_t(sizeof(T) * n);
  return ASGK_OK;
}

// the full 1D operator of every dimension (3 r1 square, row-major, row =
// output (1D cell, polynomial), column = input), from the plan's pre-summed
// 3x3 blocks
int full_1d_operators(plan_data const &p, int &r1, std::vector<std::vector<double>> &F)
{
  int const d         = p.d;
  int64_t const nconn = int64_t(p.g_conn_row.size());
  r1                  = 0;
  for (int64_t j = 0; j < nconn; j++)
    r1 = std::max(r1, std::max(p.g_conn_row[j], p.g_conn_col[j]) + 1);
  std::vector<double> B(size_t(nconn) * d * 10);
  ASGK_CUDA(cudaMemcpy(B.data(), p.gB64, sizeof(double) * B.size(), cudaMemcpyDeviceToHost));
  int const nf = 3 * r1;
  F.assign(d, std::vector<double>(size_t(nf) * nf, 0.0));
  for (int64_t j = 0; j < nconn; j++)
    for (int k = 0; k < d; k++)
    {
      const double *b = &B[size_t(j * d + k) * 10];
      int const r = p.g_conn_row[j], c = p.g_conn_col[j];
      for (int jj = 0; jj < 3; jj++)
        for (int i = 0; i < 3; i++)
          F[k][size_t(3 * r + i) * nf + 3 * c + jj] = b[i + 3 * jj];
    }
  return ASGK_OK;
}

// The class matrices in the layout the kernel's bulk copies expect: chunk j
// (columns 64 j .. 64 j + kc) is Np x kc values, row n / column kk of the
// chunk at element (n / 8) * kc * 8 + (kk / 8) * 64 + (n % 8) * 8 + kk % 8.
void class_images(std::vector<tc_class_host> const &classes, int r1,
                  std::vector<std::vector<double>> const &F, std::vector<__nv_bfloat16> &img)
{
  int const nf = 3 * r1;
  for (auto const &c : classes)
  {
    auto const &A = F[c.k];
    for (int kk0 = 0; kk0 < c.Kp; kk0 += kTcK)
    {
      int const kc      = std::min(kTcK, c.Kp - kk0);
      size_t const base = size_t(c.img_off) + size_t(c.Np) * kk0;
      for (int n = 0; n < c.Np; n++)
        for (int kl = 0; kl < kc; kl++)
        {
          int const kk = kk0 + kl;
          double v     = 0.0;
          if (n < c.R && kk < c.R)
            v = A[size_t(3 * c.set[n / 3] + n % 3) * nf + 3 * c.set[kk / 3] + kk % 3];
          size_t const e = base + size_t(n / 8) * kc * 8 + size_t(kl / 8) * 64 + (n % 8) * 8 + kl % 8;
          img[e]         = __double2bfloat16(v);
        }
    }
  }
}

// shared memory for a launch: A and B chunk buffers of the launch's widest
// chunk (K columns) and largest matrix, two of each when some matrix needs
// several chunks (double buffering), one otherwise; raised until at most
// 512 / cols CTAs fit on an SM, so the resident CTAs of one launch never ask
// for more than the SM's 512 columns.  CTAs of the concurrent launches of the
// same dimension can share an SM; a tcgen05.alloc that finds too few free
// columns then waits until a resident CTA deallocates, which every CTA does
// without waiting on any other CTA, so the wait always ends
int launch_smem(int d, tc_launch &l)
{
  int const cols = l.cols;
  int const kc   = std::min(kTcK, l.kp_max);
  l.nbuf         = l.kp_max > kTcK ? 2 : 1;
  l.abytes       = l.tpc * kTcRows * kc * 2;
  l.bbytes       = l.np_max * kc * 2;
  void *fn = tc_kernel_d(d, l.nt, l.tpc);
  size_t s = size_t(l.nbuf) * (l.abytes + l.bbytes);
  int const allowed = 512 / cols;
  int dev = 0, optin = 0;
  ASGK_CUDA(cudaGetDevice(&dev));
  ASGK_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  // the opt-in limit covers the kernel's static shared memory as well
  cudaFuncAttributes fa{};
  ASGK_CUDA(cudaFuncGetAttributes(&fa, fn));
  int const dyn_max = optin - int(fa.sharedSizeBytes);
  ASGK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max));
  for (;;)
  {
    if (s > size_t(dyn_max))
      return ASGK_ERR_UNSUPPORTED;
    int nb = 0;
    ASGK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, l.nt, s));
    if (nb >= 1 && nb <= allowed)
      break;
    if (nb < 1)
      return ASGK_ERR_UNSUPPORTED;
    s += 4096;
  }
  l.smem = s;
  return ASGK_OK;
}

} // namespace

void tc_free(tc_data *t) { delete t; }

int64_t tc_bytes(const tc_data *t) { return t != nullptr ? t->bytes : 0; }

int tc_prepare(plan_data const &p)
{
  if (p.tc != nullptr)
    return ASGK_OK;
  tc_data *t = nullptr;
  if (int rc = tc_build(p, &t))
  {
    tc_free(t);
    return rc;
  }
  p.tc = t;
  return ASGK_OK;
}

int tc_read_error(int reset, int *code)
{
  int v = 0;
  ASGK_CUDA(cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)));
  if (reset && v != 0)
  {
    int const zero = 0;
    ASGK_CUDA(cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)));
  }
  *code = v;
  return ASGK_OK;
}

int tc_build(plan_data const &p, tc_data **out)
{
  *out = nullptr;
  if (!p.global || p.gchains > 0 || p.n != 3 || p.rows != p.cols || p.d < 1 || p.d > 6)
    return ASGK_ERR_UNSUPPORTED;
  int const d = p.d;
  int r1      = 0;
  std::vector<std::vector<double>> F;
  if (int rc = full_1d_operators(p, r1, F))
    return rc;
  int const nf = 3 * r1;
  auto t       = std::make_unique<tc_data>();
  t->d = d, t->rows = p.rows, t->ts = p.tensor;
  for (int k = 0; k < d; k++)
  {
    bool nz = false;
    for (double v : F[k])
      if (v != 0.0)
      {
        nz = true;
        break;
      }
    if (nz)
      t->dims.push_back(k);
  }
  if (t->dims.empty())
    return ASGK_ERR_UNSUPPORTED;
  // every cell's 1D cells (its self connections in the diagonal pair list)
  std::vector<int> selfc(size_t(p.rows) * d), c1(size_t(p.rows) * d);
  ASGK_CUDA(cudaMemcpy(selfc.data(), p.idx, sizeof(int) * selfc.size(), cudaMemcpyDeviceToHost));
  for (size_t e = 0; e < selfc.size(); e++)
    c1[e] = p.g_conn_row[selfc[e]];
  int bits = 1;
  while ((1 << bits) < r1)
    ++bits;
  if (bits * (d - 1) > 63)
    return ASGK_ERR_UNSUPPORTED;
  // dimensions with equal operators share their class matrices
  std::vector<int> opid(d);
  for (int k = 0; k < d; k++)
  {
    opid[k] = k;
    for (int k2 = 0; k2 < k; k2++)
      if (F[k2] == F[k])
      {
        opid[k] = k2;
        break;
      }
  }
  std::map<std::pair<int, std::vector<int>>, int> class_of;
  std::vector<tc_group> groups;
  std::vector<int> pen_start, pen_cells;
  int const fib = p.tensor / 3;
  int64_t img_len = 0;
  for (int k : t->dims)
  {
    // pencils along k: cells keyed by their 1D cells outside k, ordered
    // along k within a pencil
    std::vector<std::pair<uint64_t, int>> keyed(p.rows);
    for (int c = 0; c < p.rows; c++)
    {
      uint64_t key = 0;
      for (int j = 0; j < d; j++)
        if (j != k)
          key = (key << bits) | uint64_t(c1[size_t(c) * d + j]);
      keyed[c] = {key, c};
    }
    std::sort(keyed.begin(), keyed.end(), [&](auto const &a, auto const &b) {
      if (a.first != b.first)
        return a.first < b.first;
      return c1[size_t(a.second) * d + k] < c1[size_t(b.second) * d + k];
    });
    // pencils grouped by class
    std::map<int, std::vector<std::vector<int>>> by_class;
    for (size_t s = 0; s < keyed.size();)
    {
      size_t e = s;
      while (e < keyed.size() && keyed[e].first == keyed[s].first)
        ++e;
      std::vector<int> set, cells;
      for (size_t i = s; i < e; i++)
      {
        cells.push_back(keyed[i].second);
        set.push_back(c1[size_t(keyed[i].second) * d + k]);
      }
      auto const key = std::make_pair(opid[k], set);
      auto it        = class_of.find(key);
      if (it == class_of.end())
      {
        tc_class_host ch;
        ch.k   = k;
        ch.set = set;
        ch.R   = 3 * int(set.size());
        ch.Kp  = (ch.R + 15) / 16 * 16;
        ch.Np  = ch.R <= 256 ? (ch.R + 15) / 16 * 16 : (ch.R + 31) / 32 * 32;
        if (ch.Np > 512)
          return ASGK_ERR_UNSUPPORTED; // TMEM holds 512 FP32 columns
        ch.img_off = int(img_len);
        img_len += int64_t(ch.Np) * ch.Kp;
        if (img_len > (int64_t(1) << 30))
          return ASGK_ERR_UNSUPPORTED;
        it = class_of.emplace(key, int(t->classes.size())).first;
        t->classes.push_back(std::move(ch));
      }
      by_class[it->second].push_back(std::move(cells));
      s = e;
    }
    // groups of this dimension, larger matrices first; tiles per TMEM size
    std::vector<int> cls;
    for (auto const &kv : by_class)
      cls.push_back(kv.first);
    std::sort(cls.begin(), cls.end(), [&](int a, int b) {
      return t->classes[a].R > t->classes[b].R;
    });
    std::map<int, std::vector<int2>, std::greater<int>> tiles_by_cols;
    std::map<int, int> npmax_by_cols, kpmax_by_cols;
    for (int ci : cls)
    {
      auto const &ch = t->classes[ci];
      auto const &ps = by_class[ci];
      tc_group g{};
      g.R = ch.R, g.Np = ch.Np, g.Kp = ch.Kp, g.img_off = ch.img_off;
      g.pen0 = int(pen_start.size()), g.npen = int(ps.size());
      for (auto const &cells : ps)
      {
        pen_start.push_back(int(pen_cells.size()));
        pen_cells.insert(pen_cells.end(), cells.begin(), cells.end());
      }
      int cols = 32;
      while (cols < ch.Np)
        cols *= 2;
      int const gid    = int(groups.size());
      int64_t const nr = int64_t(g.npen) * fib;
      if (nr > (int64_t(1) << 30))
        return ASGK_ERR_UNSUPPORTED;
      // matrices of up to 3 x 8 cells: four tiles per CTA
      int64_t const step = int64_t(kTcRows) * (cols == 32 ? kTcTilesSmall : 1);
      for (int64_t r0 = 0; r0 < nr; r0 += step)
        tiles_by_cols[cols].push_back(make_int2(gid, int(r0)));
      npmax_by_cols[cols] = std::max(npmax_by_cols[cols], ch.Np);
      kpmax_by_cols[cols] = std::max(kpmax_by_cols[cols], ch.Kp);
      groups.push_back(g);
    }
    for (auto &kv : tiles_by_cols)
    {
      tc_launch l;
      l.k      = k;
      l.cols   = kv.first;
      l.np_max = npmax_by_cols[kv.first];
      l.kp_max = kpmax_by_cols[kv.first];
      l.ntiles = int(kv.second.size());
      // 1-8-cell pencils: four tiles per 512-thread CTA; 16-cell pencils:
      // one tile per 128-thread CTA; larger: one tile per 512-thread CTA
      l.tpc = (kv.first == 32) ? kTcTilesSmall : 1;
      l.nt  = (kv.first == 32 || kv.first >= 128) ? kTcThreadsWide : kTcThreads;
      l.cols = 32;
      while (l.cols < l.tpc * l.np_max)
        l.cols *= 2;
      if (int rc = launch_smem(d, l))
        return rc;
      // recorded before the upload, so the destructor frees its tiles on
      // every error path
      t->launches.push_back(l);
      if (int rc = upload_tc(&t->launches.back().tiles, kv.second, t->bytes))
        return rc;
    }
  }
  pen_start.push_back(int(pen_cells.size()));
  t->img_len = img_len;
  std::vector<__nv_bfloat16> img(static_cast<size_t>(img_len));
  class_images(t->classes, r1, F, img);
  (void)nf;
  int rc;
  if ((rc = upload_tc(&t->groups, groups, t->bytes)) ||
      (rc = upload_tc(&t->pen_start, pen_start, t->bytes)) ||
      (rc = upload_tc(&t->pen_cells, pen_cells, t->bytes)) ||
      (rc = upload_tc(&t->img, img, t->bytes)))
    return rc;
  int per_dim = 0;
  for (int k : t->dims)
  {
    int c = 0;
    for (auto const &l : t->launches)
      c += (l.k == k);
    per_dim = std::max(per_dim, c);
  }
  ASGK_CUDA(cudaEventCreateWithFlags(&t->fork, cudaEventDisableTiming));
  for (int i = 1; i < per_dim; i++)
  {
    cudaStream_t st = nullptr;
    cudaEvent_t ev  = nullptr;
    ASGK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    t->side.push_back(st);
    ASGK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    t->join.push_back(ev);
  }
  int64_t const n = int64_t(p.rows) * p.tensor;
  ASGK_CUDA(cudaMalloc(&t->xb, sizeof(__nv_bfloat16) * std::max<int64_t>(n, 1)));
  ASGK_CUDA(cudaMalloc(&t->acc, sizeof(float) * std::max<int64_t>(n, 1)));
  t->bytes += int64_t(sizeof(__nv_bfloat16) + sizeof(float)) * n;
  *out = t.release();
  return ASGK_OK;
}

// new operator values (same structure): the class matrices are rewritten in
// place, so recorded launches keep their pointers
int tc_refresh(plan_data const &p, tc_data &t)
{
  int r1 = 0;
  std::vector<std::vector<double>> F;
  if (int rc = full_1d_operators(p, r1, F))
    return rc;
  std::vector<__nv_bfloat16> img(static_cast<size_t>(t.img_len));
  class_images(t.classes, r1, F, img);
  ASGK_CUDA(cudaMemcpy(t.img, img.data(), sizeof(__nv_bfloat16) * img.size(),
                       cudaMemcpyHostToDevice));
  return ASGK_OK;
}

int launch_global_tc(plan_data const &p, double alpha, const double *x, double beta,
                     double *y, double ex, cudaStream_t s)
{
  if (p.tc == nullptr)
    return ASGK_ERR_UNSUPPORTED;
  tc_data const &t = *p.tc;
  int64_t const n  = int64_t(t.rows) * t.ts;
  {
    int const blocks = int(std::min<int64_t>((n + 255) / 256, 8 * 148));
    k_to_bf16<<<blocks, 256, 0, s>>>(x, t.xb, n, g_gate);
    ASGK_LAUNCHED();
  }
  int const kfirst = t.dims.front(), klast = t.dims.back();
  size_t li = 0;
  for (int k : t.dims)
  {
    size_t le = li;
    while (le < t.launches.size() && t.launches[le].k == k)
      ++le;
    int const nl = int(le - li);
    if (nl > 1)
    {
      ASGK_CUDA(cudaEventRecord(t.fork, s));
      for (int i = 1; i < nl; i++)
        ASGK_CUDA(cudaStreamWaitEvent(t.side[i - 1], t.fork, 0));
    }
    int const mode = (kfirst == klast) ? 3 : (k == kfirst ? 0 : (k == klast ? 2 : 1));
    int const post = ipow3t(t.d - 1 - k);
    for (int i = 0; i < nl; i++)
    {
      tc_launch const &l = t.launches[li + i];
      cudaStream_t const ls = (i == 0) ? s : t.side[i - 1];
#define ASGK_TC_LAUNCH(DD, NT, TL)                                                          \
  k_tc_pencil<DD, NT, TL><<<l.ntiles, NT, l.smem, ls>>>(                                   \
      l.tiles, t.groups, t.pen_start, t.pen_cells, t.img, t.xb, t.acc, post,               \
      uint32_t(l.cols), l.abytes, l.bbytes, l.nbuf, mode, alpha, x, beta, y, ex, g_gate)
#define ASGK_TC_LAUNCH_D(DD)                                                                \
  if (l.tpc == kTcTilesSmall)                                                               \
    ASGK_TC_LAUNCH(DD, kTcThreadsWide, kTcTilesSmall);                                      \
  else if (l.nt == kTcThreadsWide)                                                          \
    ASGK_TC_LAUNCH(DD, kTcThreadsWide, 1);                                                  \
  else                                                                                      \
    ASGK_TC_LAUNCH(DD, kTcThreads, 1)
      switch (t.d)
      {
      case 1: ASGK_TC_LAUNCH_D(1); break;
      case 2: ASGK_TC_LAUNCH_D(2); break;
      case 3: ASGK_TC_LAUNCH_D(3); break;
      case 4: ASGK_TC_LAUNCH_D(4); break;
      case 5: ASGK_TC_LAUNCH_D(5); break;
      case 6: ASGK_TC_LAUNCH_D(6); break;
      default: return ASGK_ERR_UNSUPPORTED;
      }
#undef ASGK_TC_LAUNCH_D
#undef ASGK_TC_LAUNCH
      ASGK_LAUNCHED();
    }
    if (nl > 1)
      for (int i = 1; i < nl; i++)
      {
        ASGK_CUDA(cudaEventRecord(t.join[i - 1], t.side[i - 1]));
        ASGK_CUDA(cudaStreamWaitEvent(s, t.join[i - 1], 0));
      }
    li = le;
  }
  return ASGK_OK;
}

} // namespace asgk
