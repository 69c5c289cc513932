// Learned preconditioner kernels (per-cell MLP).
#include "mlp.cuh"

namespace asgk
{
int mlp_precondition(asgk_mlp *, asgk_plan *, const double *, double *,
                     cudaStream_t)
{
  return ASGK_ERR_UNSUPPORTED;
}
} // namespace asgk
