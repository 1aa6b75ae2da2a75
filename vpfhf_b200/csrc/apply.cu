// apply.cu -- instantiations of the tile engine for the U and V operators.
#include <mutex>

#include "kernels.h"
#include "ops.cuh"

namespace vfgpu {

constexpr int U_TY = 8, V_TY = 8;

cudaError_t apply_kernel_attributes() {
  static std::mutex m;  // contexts may be created from several threads
  std::lock_guard<std::mutex> lk(m);
  cudaError_t e = set_tile_attributes<UOp<double>, U_TY, 1>();
  if (e == cudaSuccess) e = set_tile_attributes<UOp<float>, U_TY, 2>();
  if (e == cudaSuccess) e = set_tile_attributes<VOp<double>, V_TY, 2>();
  if (e == cudaSuccess) e = set_tile_attributes<VOp<float>, V_TY, 3>();
  return e;
}

TilePlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms) {
  return tile_plan(nx, ny, nz, U_TY, 3, prec_bytes == 8 ? 1 : 2, num_sms);
}
TilePlan v_plan(int nx, int ny, int nz, int prec_bytes, int num_sms) {
  return tile_plan(nx, ny, nz, V_TY, 1, prec_bytes == 8 ? 2 : 3, num_sms);
}

template <>
cudaError_t launch_u_apply<double>(const UApplyArgs<double>& A, const TilePlan& p,
                                   const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<UOp<double>, U_TY, 1>(A, p, L, s);
}
template <>
cudaError_t launch_u_apply<float>(const UApplyArgs<float>& A, const TilePlan& p,
                                  const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<UOp<float>, U_TY, 2>(A, p, L, s);
}
template <>
cudaError_t launch_v_apply<double>(const VApplyArgs<double>& A, const TilePlan& p,
                                   const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<VOp<double>, V_TY, 2>(A, p, L, s);
}
template <>
cudaError_t launch_v_apply<float>(const VApplyArgs<float>& A, const TilePlan& p,
                                  const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<VOp<float>, V_TY, 3>(A, p, L, s);
}

}  // namespace vfgpu
