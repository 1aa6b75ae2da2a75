// apply.cu -- instantiations of the tile engine for the U and V operators.
#include <mutex>
#include <type_traits>

#include "kernels.h"
#include "ops.cuh"

namespace vfgpu {

// FP64 U operator tiles: 32 x U64_TY elements (1 CTA per SM: ~250 registers per thread).
// 12 rows (12 warps per SM at 168 registers, with 288 bytes of spills) measured slower
// on B200: 0.280 against 0.253 ms at 129^3, 0.814 against 0.733 ms at 193^3.
#ifndef VFGPU_U64_TY
#define VFGPU_U64_TY 8
#endif
constexpr int U_TY = 8, U64_TY = VFGPU_U64_TY, V_TY = kVTileY;
// Blocks per SM of the FP64 U operator: 1 (~250 registers, two corner-contribution
// buffers) or, as a build option, 2 (128 registers: the row closed form of the
// non-constant elements spills; one buffer and a second barrier per layer).
#ifndef VFGPU_U64_MINB
#define VFGPU_U64_MINB 1
#endif
constexpr int U64_MINB = VFGPU_U64_MINB;
// V tiles carry 2 stages of 27 coefficients per cell in shared memory: 75 KB (FP32,
// 2 CTAs per SM) or 150 KB (FP64, 1 CTA per SM).
constexpr int V64_MINB = 1, V32_MINB = 2;
// FP32 U operator: scalar UOp<float> (2 CTAs of 8 warps per SM) by default.  The
// packed two-lane variant (UOpF2: two elements per thread, half the arithmetic
// instructions) is kept as a build option; it needs 242 registers, so one CTA of
// 8 warps per SM, and measured slower on B200: 0.185 ms against 0.161 ms at 129^3,
// 0.353 ms against 0.298 ms at 161^3 (16 element rows; 0.189 / 0.339 ms with 8).
#ifndef VFGPU_U32_PACKED
#define VFGPU_U32_PACKED 0
#endif
#ifndef VFGPU_U32_PACKED_TY
#define VFGPU_U32_PACKED_TY 16
#endif
constexpr bool kU32Packed = VFGPU_U32_PACKED != 0;
constexpr int U32_TY = kU32Packed ? VFGPU_U32_PACKED_TY : U_TY;
#ifndef VFGPU_U32_MINB
#define VFGPU_U32_MINB 2
#endif
constexpr int U32_MINB = kU32Packed ? (VFGPU_U32_PACKED_TY == 16 ? 1 : 2) : VFGPU_U32_MINB;
using U32Op = std::conditional_t<kU32Packed, UOpF2, UOp<float>>;
using U32OpC = std::conditional_t<kU32Packed, UOpF2, UOp<float, true>>;

// Cubic cells take the U element with every 1/h folded into the row weight.
template <typename T> bool cubic(const UApplyArgs<T>& A) { return A.ihx == A.ihy && A.ihy == A.ihz; }

cudaError_t apply_kernel_attributes() {
  static std::mutex m;  // contexts may be created from several threads
  std::lock_guard<std::mutex> lk(m);
  cudaError_t e = set_tile_attributes<UOp<double>, U64_TY, U64_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<UOp<double, true>, U64_TY, U64_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<U32Op, U32_TY, U32_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<U32OpC, U32_TY, U32_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<UOpNC<double>, U64_TY, 1>();
  if (e == cudaSuccess) e = set_tile_attributes<UOpNC<float>, U_TY, 2>();
  if (e == cudaSuccess) e = set_tile_attributes<VOp<double>, V_TY, V64_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<VOp<float>, V_TY, V32_MINB>();
  return e;
}

cudaError_t vcoef_tensor_map(CUtensorMap* map, const void* coef, int bytes, int nex, int ney, int nez) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                              CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                              CUtensorMapFloatOOBfill);
  static const Encode encode = []() -> Encode {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<Encode>(fn);
  }();
  if (!encode) return cudaErrorNotSupported;
  const int pitch = vcoef_pitch(nex);
  const cuuint64_t dims[3] = {(cuuint64_t)nex, (cuuint64_t)ney, (cuuint64_t)27 * nez};
  const cuuint64_t strides[2] = {(cuuint64_t)pitch * bytes, (cuuint64_t)pitch * ney * bytes};
  const cuuint32_t box[3] = {32, (cuuint32_t)kVTileY, 27}, estride[3] = {1, 1, 1};
  const CUresult r =
      encode(map, bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
             const_cast<void*>(coef), dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// One CTA waits on an mbarrier whose phase completes (complete = 1: the arrival is
// made) or never does (complete = 0: 16 transaction bytes are expected and no copy is
// issued); the bounded wait sets *err when it gives up.
__global__ void wait_selftest_kernel(unsigned* err, long long limit, int complete) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
    if (complete) mbar_arrive(&bar);
    else mbar_expect_tx(&bar, 16);
  }
  __syncthreads();
  mbar_wait(&bar, 0, err, limit);
}

cudaError_t wait_selftest(long long cycles, int complete, int* timed_out) {
  unsigned* d = nullptr;
  unsigned h = 0;
  cudaError_t e = cudaMalloc(&d, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(unsigned));
  if (e == cudaSuccess) {
    wait_selftest_kernel<<<1, 64>>>(d, cycles, complete);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost);
  cudaFree(d);
  *timed_out = h ? 1 : 0;
  return e;
}

TilePlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms) {
  if (prec_bytes == 8) return tile_plan(nx, ny, nz, U64_TY, 3, U64_MINB, num_sms);
  return tile_plan(nx, ny, nz, U32_TY, 3, U32_MINB, num_sms);
}
TilePlan v_plan(int nx, int ny, int nz, int prec_bytes, int num_sms) {
  return tile_plan(nx, ny, nz, V_TY, 1, prec_bytes == 8 ? V64_MINB : V32_MINB, num_sms);
}

template <>
cudaError_t launch_u_apply<double>(const UApplyArgs<double>& A, const TilePlan& p,
                                   const LayerTable& L, cudaStream_t s) {
  if (A.cflag) return launch_tile_apply<UOpNC<double>, U64_TY, 1>(A, p, L, s);
  if (cubic(A)) return launch_tile_apply<UOp<double, true>, U64_TY, U64_MINB>(A, p, L, s);
  return launch_tile_apply<UOp<double>, U64_TY, U64_MINB>(A, p, L, s);
}
template <>
cudaError_t launch_u_apply<float>(const UApplyArgs<float>& A, const TilePlan& p,
                                  const LayerTable& L, cudaStream_t s) {
  // NOCOMPRESSION needs the scalar layout: its plan is the FP32 plan only with the
  // scalar tile (the packed build option keeps the plain operator packed)
  if (A.cflag) return launch_tile_apply<UOpNC<float>, U_TY, 2>(A, p, L, s);
  if (cubic(A)) return launch_tile_apply<U32OpC, U32_TY, U32_MINB>(A, p, L, s);
  return launch_tile_apply<U32Op, U32_TY, U32_MINB>(A, p, L, s);
}
template <>
cudaError_t launch_v_apply<double>(const VApplyArgs<double>& A, const TilePlan& p,
                                   const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<VOp<double>, V_TY, V64_MINB>(A, p, L, s);
}
template <>
cudaError_t launch_v_apply<float>(const VApplyArgs<float>& A, const TilePlan& p,
                                  const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<VOp<float>, V_TY, V32_MINB>(A, p, L, s);
}

}  // namespace vfgpu

extern "C" int vfgpu_wait_selftest(long long cycles, int complete, int* timed_out) {
  if (!timed_out || cycles < 0 || cycles > 4000000000ll) return -1;
  return vfgpu::wait_selftest(cycles, complete ? 1 : 0, timed_out) == cudaSuccess ? 0 : -2;
}
