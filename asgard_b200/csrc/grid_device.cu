// Connected cell pairs of a sparse grid built on the device (operator setup;
// the host builder in grid.cpp computes the same list).
//
// The reference's rule (check_connected, src/asgard_kronmult_matrix.cpp:
// 230-300; the pair list of make_kronmult_sparse, :406-466): two cells are
// connected when their 1D cells are connected in every dimension.  One CTA
// per output cell tests every candidate cell against the 1D connection
// table (the connection's index, or -1) -- the brute-force pass the
// reference runs on the host, here at a few milliseconds for 2.6e8 pairs --
// first counting, then writing each row's pairs in candidate order (a
// warp-ballot prefix per chunk of candidates, so the order is the
// candidates' whatever the scheduling) with the d connection indices.
#include "internal.cuh"

namespace asgk
{
namespace
{
constexpr int kPairThreads = 256;
constexpr int kPairWarps   = kPairThreads / 32;

template<int D>
__global__ void __launch_bounds__(kPairThreads)
    k_count_pairs(int cells, const int *__restrict__ oned,
                  const int *__restrict__ cand, const int *__restrict__ lut,
                  int R, int64_t *__restrict__ counts)
{
  __shared__ int warp_cnt[kPairWarps];
  int const r = blockIdx.x;
  int ro[D];
#pragma unroll
  for (int k = 0; k < D; k++)
    ro[k] = __ldg(oned + int64_t(r) * D + k) * R;
  int cnt = 0;
  for (int i = threadIdx.x; i < cells; i += kPairThreads)
  {
    int const c = __ldg(cand + i);
    bool ok     = true;
#pragma unroll
    for (int k = 0; k < D; k++)
      ok = ok && __ldg(lut + ro[k] + __ldg(oned + int64_t(c) * D + k)) >= 0;
    cnt += ok ? 1 : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0)
    warp_cnt[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    int64_t s = 0;
    for (int w = 0; w < kPairWarps; w++)
      s += warp_cnt[w];
    counts[r] = s;
  }
}

template<int D>
__global__ void __launch_bounds__(kPairThreads)
    k_fill_pairs(int cells, const int *__restrict__ oned,
                 const int *__restrict__ cand, const int *__restrict__ lut,
                 int R, const int64_t *__restrict__ row_ptr,
                 int *__restrict__ col, int *__restrict__ conn)
{
  __shared__ int warp_tot[kPairWarps];
  __shared__ int warp_off[kPairWarps + 1];
  int const r    = blockIdx.x;
  int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int ro[D];
#pragma unroll
  for (int k = 0; k < D; k++)
    ro[k] = __ldg(oned + int64_t(r) * D + k) * R;
  int64_t pos = row_ptr[r];
  for (int chunk = 0; chunk < cells; chunk += kPairThreads)
  {
    int const i = chunk + threadIdx.x;
    bool ok     = false;
    int c       = 0;
    int jj[D];
    if (i < cells)
    {
      c  = __ldg(cand + i);
      ok = true;
#pragma unroll
      for (int k = 0; k < D; k++)
      {
        jj[k] = __ldg(lut + ro[k] + __ldg(oned + int64_t(c) * D + k));
        ok    = ok && jj[k] >= 0;
      }
    }
    unsigned const m = __ballot_sync(0xffffffffu, ok);
    if (lane == 0)
      warp_tot[warp] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0)
    {
      int s = 0;
      for (int w = 0; w < kPairWarps; w++)
      {
        warp_off[w] = s;
        s += warp_tot[w];
      }
      warp_off[kPairWarps] = s;
    }
    __syncthreads();
    if (ok)
    {
      int64_t const p = pos + warp_off[warp] + __popc(m & ((1u << lane) - 1u));
      col[p]          = c;
#pragma unroll
      for (int k = 0; k < D; k++)
        conn[p * D + k] = jj[k];
    }
    pos += warp_off[kPairWarps];
    __syncthreads(); // warp_tot / warp_off are rewritten by the next chunk
  }
}

template<int D>
int count_d(int cells, const int *oned, const int *cand, const int *lut, int R,
            int64_t *counts, cudaStream_t s)
{
  k_count_pairs<D><<<cells, kPairThreads, 0, s>>>(cells, oned, cand, lut, R, counts);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

template<int D>
int fill_d(int cells, const int *oned, const int *cand, const int *lut, int R,
           const int64_t *row_ptr, int *col, int *conn, cudaStream_t s)
{
  k_fill_pairs<D><<<cells, kPairThreads, 0, s>>>(cells, oned, cand, lut, R,
                                                 row_ptr, col, conn);
  ASGK_LAUNCHED();
  return ASGK_OK;
}

} // namespace

int launch_count_pairs(int d, int cells, const int *oned, const int *cand,
                       const int *lut, int R, int64_t *counts, cudaStream_t s)
{
  if (cells <= 0)
    return ASGK_OK;
  switch (d)
  {
  case 1: return count_d<1>(cells, oned, cand, lut, R, counts, s);
  case 2: return count_d<2>(cells, oned, cand, lut, R, counts, s);
  case 3: return count_d<3>(cells, oned, cand, lut, R, counts, s);
  case 4: return count_d<4>(cells, oned, cand, lut, R, counts, s);
  case 5: return count_d<5>(cells, oned, cand, lut, R, counts, s);
  case 6: return count_d<6>(cells, oned, cand, lut, R, counts, s);
  default: return ASGK_ERR_UNSUPPORTED;
  }
}

int launch_fill_pairs(int d, int cells, const int *oned, const int *cand,
                      const int *lut, int R, const int64_t *row_ptr, int *col,
                      int *conn, cudaStream_t s)
{
  if (cells <= 0)
    return ASGK_OK;
  switch (d)
  {
  case 1: return fill_d<1>(cells, oned, cand, lut, R, row_ptr, col, conn, s);
  case 2: return fill_d<2>(cells, oned, cand, lut, R, row_ptr, col, conn, s);
  case 3: return fill_d<3>(cells, oned, cand, lut, R, row_ptr, col, conn, s);
  case 4: return fill_d<4>(cells, oned, cand, lut, R, row_ptr, col, conn, s);
  case 5: return fill_d<5>(cells, oned, cand, lut, R, row_ptr, col, conn, s);
  case 6: return fill_d<6>(cells, oned, cand, lut, R, row_ptr, col, conn, s);
  default: return ASGK_ERR_UNSUPPORTED;
  }
}

} // namespace asgk
