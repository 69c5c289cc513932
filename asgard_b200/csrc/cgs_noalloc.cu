// asgk_cgs_step_noalloc: the Gram-Schmidt step of asgk_cgs_step without any
// device allocation.
//
// Who needs it: callers that must not allocate device memory once their solve
// is running -- a time-stepping code that handed all free device memory to its
// own pool at start-up (so cudaMalloc would fail or fragment it), or a caller
// that cannot afford the device-wide synchronisation cudaMalloc/cudaFree
// imply, or one whose memory pools are disabled so stream-ordered allocation
// is not available.  They still pass their own inputs and outputs (V, w, h);
// only the partial sums of the reductions, which asgk_cgs_step allocates per
// call, come from a fixed array compiled into this library.
//
// Limits and rules:
//   * k <= kMaxK (256) columns, and at most kMaxBlocks (512)
//     reduction blocks (2 per SM, so GPUs with up to 256 SMs); larger requests
//     return ASGK_ERR_NOALLOC_LIMIT without touching any argument;
//   * the array (kScratch doubles, 1 MiB) exists on every GPU that loads
//     the library and is held until the process exits;
//   * every call writes the partial sums it later reads, so nothing has to
//     start at zero, but all calls on a device share the one array: calls that
//     overlap on the GPU (e.g. on two streams) race and must be serialised by
//     the caller;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and caches it; make that
//     first call before any stream capture.
#include "internal.cuh"

#include <cmath>
#include <mutex>

namespace
{
constexpr int kMaxK      = 256;
constexpr int kMaxBlocks = 512;
// the multi-dot pass writes one partial sum per (block, column), at most
// kMaxBlocks * kMaxK; the norm pass then reuses the start of that region for
// its kMaxBlocks partials, and their sum goes to the slot after it
constexpr size_t kNormSlot = size_t(kMaxBlocks) * kMaxK;
constexpr size_t kScratch  = kNormSlot + 1;
} // namespace

// The scratch itself.  In host code this name is only a stand-in for the
// device symbol: host code must use the address from cudaGetSymbolAddress.
static __device__ __align__(256) double g_cgs_scratch[kScratch];

namespace
{
constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of g_cgs_scratch on the current device (looked up once).
int scratch_address(double **out)
{
  int dev = 0;
  ASGK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return ASGK_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr)
  {
    void *p = nullptr;
    cudaError_t const e = cudaGetSymbolAddress(&p, g_cgs_scratch);
    if (e != cudaSuccess || p == nullptr)
    {
      std::fprintf(stderr,
                   "asgard_b200: cudaGetSymbolAddress of the no-alloc scratch "
                   "failed on device %d: %s\n",
                   dev, cudaGetErrorString(e));
      return ASGK_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return ASGK_OK;
}
} // namespace

namespace
{
int cgs_step_noalloc(const double *V, int64_t ldv, int k, double *w, int64_t n,
                     double *h, double *norm, asgk_stream stream)
{
  using namespace asgk;
  if (!V || !w || !h || !norm || k < 1 || n < 1 || ldv < n)
    return ASGK_ERR_INVALID;
  if (k > kMaxK)
  {
    std::fprintf(stderr,
                 "asgard_b200: asgk_cgs_step_noalloc: k = %d columns exceeds "
                 "the fixed scratch limit of %d\n",
                 k, kMaxK);
    return ASGK_ERR_NOALLOC_LIMIT;
  }
  if (max_reduction_blocks() > kMaxBlocks)
  {
    std::fprintf(stderr,
                 "asgard_b200: asgk_cgs_step_noalloc: %d reduction blocks "
                 "exceed the fixed scratch limit of %d\n",
                 max_reduction_blocks(), kMaxBlocks);
    return ASGK_ERR_NOALLOC_LIMIT;
  }
  double *part = nullptr;
  if (int rc = scratch_address(&part))
    return rc;
  double *nrm2   = part + kNormSlot;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int used       = 0;
  if (int rc = launch_multidot(V, ldv, k, w, n, part, &used, s))
    return rc;
  if (int rc = launch_reduce_parts(part, used, k, h, s))
    return rc;
  if (int rc = launch_update_norm(V, ldv, k, h, w, n, part, &used, s))
    return rc;
  if (int rc = launch_reduce_parts(part, used, 1, nrm2, s))
    return rc;
  double host = 0;
  ASGK_CUDA(cudaMemcpyAsync(&host, nrm2, sizeof(double),
                            cudaMemcpyDeviceToHost, s));
  ASGK_CUDA(cudaStreamSynchronize(s));
  *norm = std::sqrt(host);
  return ASGK_OK;
}
} // namespace

// As every status-returning entry of the C ABI, no host exception crosses
// the boundary (the mutex of the address cache can throw std::system_error).
extern "C" int asgk_cgs_step_noalloc(const double *V, int64_t ldv, int k,
                                     double *w, int64_t n, double *h,
                                     double *norm, asgk_stream stream)
{
  try
  {
    return cgs_step_noalloc(V, ldv, k, w, n, h, norm, stream);
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
