// kernels.h -- host-side declarations of the vfgpu kernel launchers.
#pragma once

#include <algorithm>

#include "common.cuh"
#include "ops.cuh"

namespace vfgpu {

cudaError_t apply_kernel_attributes();
TilePlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms);
TilePlan v_plan(int nx, int ny, int nz, int prec_bytes, int num_sms);
// Element rows of a V tile: the y extent of the coefficient tensor copy's box.
constexpr int kVTileY = 8;
// The V coefficient array (vcoef_index layout, 8- or 4-byte values) as the 3-D tensor
// the V apply stages from: box 32 x kVTileY x 27.
cudaError_t vcoef_tensor_map(CUtensorMap* map, const void* coef, int bytes, int nex, int ney, int nez);
// The bounded mbarrier wait of the tensor-copy pipeline, alone: *timed_out = 1 when a
// wait on a phase that never completes (complete = 0) gave up after `cycles`.
cudaError_t wait_selftest(long long cycles, int complete, int* timed_out);

template <typename T>
cudaError_t launch_u_apply(const UApplyArgs<T>& A, const TilePlan& p, const LayerTable& L,
                           cudaStream_t s);
template <typename T>
cudaError_t launch_v_apply(const VApplyArgs<T>& A, const TilePlan& p, const LayerTable& L,
                           cudaStream_t s);

}  // namespace vfgpu
