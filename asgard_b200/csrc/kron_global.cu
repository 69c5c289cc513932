// Global-mode kronmult apply (n = 3): the operator of terms that act in one
// dimension each, applied through the cell pairs that differ in at most one
// dimension.
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

namespace asgk
{
namespace
{
constexpr int ipow3g(int k) { return k == 0 ? 1 : 3 * ipow3g(k - 1); }

template<typename TC> struct padG;
template<> struct padG<double> { static constexpr int value = 10; };
template<> struct padG<float> { static constexpr int value = 12; };

// One CTA per output cell.  The cell's neighbour list is staged in shared
// memory (coalesced, CAP entries at a time) so that the neighbours' tensor
// loads do not wait on their indices; the NW warps take the entries in turn,
// four in flight per warp, each warp holding a partial output tensor (PER
// entries per lane), summed over the warps in shared memory at the end.
template<int D, typename TC, int NW>
__global__ void __launch_bounds__(NW * 32)
    kron_global_rows(const int64_t *__restrict__ gptr,
                     const int *__restrict__ gcol, const int *__restrict__ gkb,
                     const TC *__restrict__ B, const int *__restrict__ row_order,
                     double alpha, const double *__restrict__ x, double beta,
                     double *__restrict__ y, double ex)
{
  constexpr int TS  = ipow3g(D);
  constexpr int PER = (TS + 31) / 32; // outputs per lane
  constexpr int PAD = padG<TC>::value;
  constexpr int CAP = 512;
  constexpr int NT  = NW * 32;
  extern __shared__ __align__(16) unsigned char smem_g[];
  TC *red    = reinterpret_cast<TC *>(smem_g);          // [NW][TS]
  int *s_col = reinterpret_cast<int *>(red + NW * TS);  // [CAP]
  int *s_kb  = s_col + CAP;                             // [CAP]

  int const warp     = threadIdx.x >> 5;
  int const lane     = threadIdx.x & 31;
  int const row      = row_order[blockIdx.x];
  int64_t const ebeg = gptr[row];
  int64_t const eend = gptr[row + 1];

  TC acc[PER];
#pragma unroll
  for (int o = 0; o < PER; o++)
    acc[o] = TC(0);

  auto entry = [&](int j) {
    int const c  = s_col[j];
    int const kb = s_kb[j];
    int const k  = kb % D;
    const TC *b  = B + int64_t(kb) * PAD;
    const double *xc = x + int64_t(c) * TS;
    int stride = 1; // of dimension k in the tensor (dimension 0 slowest)
#pragma unroll
    for (int q = D - 1; q > 0; q--)
      if (q > k)
        stride *= 3;
#pragma unroll
    for (int o = 0; o < PER; o++)
    {
      int const i = lane + 32 * o;
      if (i < TS)
      {
        int const ik   = (i / stride) % 3;
        int const base = i - ik * stride;
        // row ik of the column-major block: b[ik + 3 j]
        TC const v0 = static_cast<TC>(__ldg(xc + base));
        TC const v1 = static_cast<TC>(__ldg(xc + base + stride));
        TC const v2 = static_cast<TC>(__ldg(xc + base + 2 * stride));
        acc[o] = fma(__ldg(b + ik + 6), v2,
                     fma(__ldg(b + ik + 3), v1, fma(__ldg(b + ik), v0, acc[o])));
      }
    }
  };
  for (int64_t cb = ebeg; cb < eend; cb += CAP)
  {
    int const n = int((eend - cb < CAP) ? (eend - cb) : CAP);
    __syncthreads(); // the previous chunk's entries are consumed
    for (int i = threadIdx.x; i < n; i += NT)
    {
      s_col[i] = __ldg(gcol + cb + i);
      s_kb[i]  = __ldg(gkb + cb + i);
    }
    __syncthreads();
    for (int j = warp; j < n; j += 4 * NW)
    {
      entry(j);
      if (j + NW < n)
        entry(j + NW);
      if (j + 2 * NW < n)
        entry(j + 2 * NW);
      if (j + 3 * NW < n)
        entry(j + 3 * NW);
    }
  }
#pragma unroll
  for (int o = 0; o < PER; o++)
  {
    int const i = lane + 32 * o;
    if (i < TS)
      red[warp * TS + i] = acc[o];
  }
  __syncthreads();
  int64_t const base = int64_t(row) * TS;
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
}

template<int D, typename TC>
int launch_global_d(plan_data const &p, double alpha, const double *x,
                    double beta, double *y, double ex, cudaStream_t s)
{
  constexpr int TS = ipow3g(D);
  constexpr int NW = TS <= 27 ? 4 : 8;
  size_t const shm = size_t(NW) * TS * sizeof(TC) + 2 * 512 * sizeof(int);
  const TC *B;
  if constexpr (sizeof(TC) == 8)
    B = p.gB64;
  else
    B = p.gB32;
  auto kern = kron_global_rows<D, TC, NW>;
  static bool configured = false;
  if (!configured)
  {
    ASGK_CUDA(cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
    configured = true;
  }
  kern<<<p.rows, NW * 32, shm, s>>>(p.gptr, p.gcol, p.gkb, B, p.row_order,
                                    alpha, x, beta, y, ex);
  ASGK_LAUNCHED();
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
  if (p.n != 3)
    return ASGK_ERR_UNSUPPORTED;
  // terms that are the identity in every dimension add n_identity * x
  double const ex_eff = ex + alpha * p.g_identity;
  if (precision == ASGK_FP64)
    return launch_global_t<double>(p, alpha, x, beta, y, ex_eff, s);
  if (precision == ASGK_FP32)
    return launch_global_t<float>(p, alpha, x, beta, y, ex_eff, s);
  return ASGK_ERR_UNSUPPORTED;
}

} // namespace asgk
