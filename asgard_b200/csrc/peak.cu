// Measured FP64 / FP32 FMA throughput of this GPU (the denominator of the
// FP64-pipe roofline of the kronmult kernels).  Each thread runs 8
// independent FMA chains; the grid covers every SM several times.
#include "internal.cuh"

#include <algorithm>

namespace asgk
{
namespace
{
template<typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T *out, int iters, T a, T b)
{
  T v[8];
#pragma unroll
  for (int i = 0; i < 8; i++)
    v[i] = T(threadIdx.x + i);
  for (int it = 0; it < iters; it++)
  {
#pragma unroll
    for (int r = 0; r < 16; r++)
    {
#pragma unroll
      for (int i = 0; i < 8; i++)
        v[i] = v[i] * a + b;
    }
  }
  T s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++)
    s += v[i];
  if (s == T(12345.678)) // never true for the inputs used; keeps the work live
    out[0] = s;
}

template<typename T>
int measure(double *tflops, int iters)
{
  int dev = 0, sms = 0;
  ASGK_CUDA(cudaGetDevice(&dev));
  ASGK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  T *out = nullptr;
  ASGK_CUDA(cudaMalloc(&out, sizeof(T)));
  cudaEvent_t e0, e1;
  ASGK_CUDA(cudaEventCreate(&e0));
  ASGK_CUDA(cudaEventCreate(&e1));
  int const blocks = sms * 8;
  k_fma_peak<T><<<blocks, 256>>>(out, iters / 4, T(0.999999), T(1e-7)); // warm-up
  ASGK_LAUNCHED();
  double const flop = 2.0 * 8 * 16 * double(iters) * blocks * 256;
  double best = 0;
  for (int rep = 0; rep < 5; rep++) // best of 5 launches
  {
    ASGK_CUDA(cudaEventRecord(e0));
    k_fma_peak<T><<<blocks, 256>>>(out, iters, T(0.999999), T(1e-7));
    ASGK_LAUNCHED();
    ASGK_CUDA(cudaEventRecord(e1));
    ASGK_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    ASGK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = std::max(best, flop / (ms * 1e-3) / 1e12);
  }
  *tflops = best;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return ASGK_OK;
}
} // namespace
} // namespace asgk

extern "C" int asgk_measure_fma_peak(int precision, double *tflops)
{
  if (!tflops)
    return ASGK_ERR_INVALID;
  if (precision == ASGK_FP64)
    return asgk::measure<double>(tflops, 4096);
  if (precision == ASGK_FP32)
    return asgk::measure<float>(tflops, 8192);
  return ASGK_ERR_UNSUPPORTED;
}
