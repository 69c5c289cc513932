// Device-side Givens update of the recorded GMRES cycles, shared by the
// Gram-Schmidt kernel that performs it (krylov.cu) and the solver that
// records the cycles (capi.cu).
#pragma once

#include "internal.cuh"

namespace asgk
{
// Device state of a recorded cycle (doubles): the estimated residual, 1/||w||
// for the new basis vector, ||w||, steps done, status, tolerance, go (1 while
// the cycle continues: the gate of the kernels of later steps); then g, the
// cosines, the sines (restart + 1 each) and the packed Hessenberg columns
// (restart*(restart+1)/2).
constexpr int kGoSlot    = 6;
constexpr int kStateHead = 7;
inline int64_t state_len(int restart)
{
  return kStateHead + 3 * int64_t(restart + 1) + int64_t(restart) * (restart + 1) / 2;
}

// Where step i of a recorded cycle reports (the Givens part of the
// update-and-norm pass): null for a host-driven step.  has_next: the step
// ends its graph node and sets the condition of the next node.
struct givens_args
{
  double *state = nullptr;
  int step      = 0;
  int restart   = 0;
  cudaGraphConditionalHandle next = 0; // condition of the next node
  int has_next  = 0;
};

// The host loop's rot / rotg (reference BLAS drotg) with round-to-nearest
// intrinsics, so that no multiply-add is contracted and the recorded cycle
// gives the host-driven cycle's rotations bit for bit.
__device__ __forceinline__ void rot_d(double &x, double &y, double c, double s)
{
  double const tx = __dadd_rn(__dmul_rn(c, x), __dmul_rn(s, y));
  double const ty = __dsub_rn(__dmul_rn(c, y), __dmul_rn(s, x));
  x = tx;
  y = ty;
}

__device__ __forceinline__ void rotg_d(double &a, double &b, double &c, double &s)
{
  double const sa = a, sb = b;
  double const roe   = (fabs(sa) > fabs(sb)) ? sa : sb;
  double const scale = __dadd_rn(fabs(sa), fabs(sb));
  double r, z;
  if (scale == 0)
  {
    c = 1;
    s = 0;
    r = 0;
    z = 0;
  }
  else
  {
    double const qa = __ddiv_rn(sa, scale), qb = __ddiv_rn(sb, scale);
    r = __dmul_rn(scale, __dsqrt_rn(__dadd_rn(__dmul_rn(qa, qa), __dmul_rn(qb, qb))));
    r = (roe >= 0) ? r : -r;
    c = __ddiv_rn(sa, r);
    s = __ddiv_rn(sb, r);
    z = 1;
    if (fabs(sa) > fabs(sb))
      z = s;
    if (fabs(sb) >= fabs(sa) && c != 0)
      z = __ddiv_rn(1.0, c);
  }
  a = r;
  b = z;
}

// Step ga.step's Givens update (one thread): hk = the projections h[0..k)
// (k = step + 1), nrm2 = ||w||^2; csn holds the cosines then the sines of the
// earlier steps (restart + 1 each, a copy in shared memory).  Writes the new
// Hessenberg column, rotation, g entries, residual estimate, 1/||w||, the go
// flag and, at the end of a node, the condition of the next node (go on
// while the estimate is above the tolerance, the cycle is not full and w is
// not zero).
__device__ __forceinline__ void givens_step(givens_args const &ga,
                                            const double *hk, double nrm2,
                                            double *coeffs, const double *csn)
{
  double *st       = ga.state;
  int const i      = ga.step;
  int const k      = i + 1;
  double *g        = st + kStateHead;
  double *cs       = g + ga.restart + 1;
  double *sn       = cs + ga.restart + 1;
  double *H        = sn + ga.restart + 1;
  double const nrm = __dsqrt_rn(nrm2);
  double const tol = st[5];
  st[2]            = nrm;
  st[3]            = k;
  unsigned go      = 0;
  if (!isfinite(nrm))
  {
    st[4] = ASGK_ERR_NONFINITE;
    st[1] = 1.0;
  }
  else
  {
    st[1] = (nrm > 0) ? 1.0 / nrm : 1.0;
    for (int j = 0; j < k; j++)
      coeffs[j] = hk[j];
    for (int j = 0; j < i; j++)
      rot_d(coeffs[j], coeffs[j + 1], csn[j], csn[ga.restart + 1 + j]);
    double beta = nrm, c = 0, s = 0;
    rotg_d(coeffs[i], beta, c, s);
    cs[i] = c;
    sn[i] = s;
    double *Hc = H + int64_t(i) * (i + 1) / 2;
    for (int j = 0; j < k; j++)
      Hc[j] = coeffs[j];
    double const res = fabs(__dmul_rn(s, g[i]));
    st[0]            = res;
    if (res > tol)
    {
      double gi = g[i], gn = 0.0;
      rot_d(gi, gn, c, s);
      g[i]     = gi;
      g[i + 1] = gn;
    }
    go = (res > tol && k < ga.restart && nrm != 0.0) ? 1u : 0u;
  }
  st[kGoSlot] = go ? 1.0 : 0.0;
  if (ga.has_next)
    cudaGraphSetConditional(ga.next, go);
}

} // namespace asgk
