// kernels.h -- host-side declarations of the vfgpu kernel launchers.
#pragma once

#include <algorithm>

#include "common.cuh"
#include "u_apply.cuh"

namespace vfgpu {

// Launch plan of the U apply: xy tiles of 32 x ty elements, z-chunks of zc planes,
// seam buffer sizes (elements of the working precision).
struct UPlan {
  int ty, ntx, nty, zc, nzc;
  size_t seamX, seamY;
};

UPlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms);

template <typename T>
cudaError_t launch_u_apply(const UApplyArgs<T>& A, const UPlan& p, const LayerTable& L,
                           cudaStream_t s);

}  // namespace vfgpu
