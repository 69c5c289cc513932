// Learned preconditioner (per-cell MLP) used inside flexible GMRES.
#pragma once

#include "internal.cuh"

namespace asgk
{
// z = M(v): applies the network cell by cell to the FP64 Krylov vector v
// (plus its base preconditioner, from its FP32 copy when low is set).
int mlp_precondition(asgk_mlp *mlp, asgk_plan *plan, const double *v,
                     double *z, cudaStream_t s, bool low);
// ASGK_OK when the network applies to rows cells of tensor values each
int mlp_check_shape(const asgk_mlp *mlp, int rows, int tensor);
} // namespace asgk
