// kernels.h -- host-side declarations of the vfgpu kernel launchers.
#pragma once

#include <algorithm>

#include "common.cuh"
#include "ops.cuh"

namespace vfgpu {

cudaError_t apply_kernel_attributes();
TilePlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms);
TilePlan v_plan(int nx, int ny, int nz, int prec_bytes, int num_sms);

template <typename T>
cudaError_t launch_u_apply(const UApplyArgs<T>& A, const TilePlan& p, const LayerTable& L,
                           cudaStream_t s);
template <typename T>
cudaError_t launch_v_apply(const VApplyArgs<T>& A, const TilePlan& p, const LayerTable& L,
                           cudaStream_t s);

}  // namespace vfgpu
