// common.cuh -- shared helpers for the vfgpu kernels (sm_100a).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vfgpu {

// 1-D 3-point Gauss rule on the reference interval t in [-1/2, 1/2]
// (VFCartFE.c:100-107: nodes (1 -+ sqrt(3/5))/2 on [0,1], weights 5/18, 8/18, 5/18).
#define VF_TAU 0.38729833462074168852   /* sqrt(3/5)/2 */
#define VF_W0 0.27777777777777777778    /* 5/18 */
#define VF_W1 0.44444444444444444444    /* 8/18 */

// Element-layer material table (per-layer VFMatProp, VFCommon.h:69-80).
#define VF_MAXLAYER 16
struct LayerTable {
  double lambda[VF_MAXLAYER];   // Lame lambda (VFCommon.c:584)
  double mu[VF_MAXLAYER];       // Lame mu     (VFCommon.c:585)
  double lamfac[VF_MAXLAYER];   // lambda / E  (for per-cell E)
  double mufac[VF_MAXLAYER];    // mu / E
  double alpha[VF_MAXLAYER];    // thermal expansion
  double beta[VF_MAXLAYER];     // Biot coefficient
  double Gc[VF_MAXLAYER];
};

// Per-problem parameters the operator kernels read through a device pointer, so
// that captured CUDA graphs stay valid when a ctx is re-used for another problem
// (set-up calls rewrite this block instead of the kernels' by-value arguments).
struct DevParams {
  LayerTable L;
  double eta;                  // eta (VFProp.eta)
  double aeps[VF_MAXLAYER];    // Gc/(2 c_w) * eps per layer (V operator gradient term)
};

template <typename T> struct Vec3 { T x, y, z; };

__host__ __device__ inline int64_t node_index(int i, int j, int k, int nx, int ny) {
  return ((int64_t)k * ny + j) * nx + i;
}

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

// The V coupling coefficient (27 Gauss-point values per cell) is stored per element
// layer as 27 planes of the layer's cells, [ez][g][ey][ex], with rows padded to a
// multiple of 4 cells (16-byte row strides, the tensor-copy rule), so that the 27
// values of a 32 x TY tile of cells are one box of a 3-D tensor copy.
__host__ __device__ inline int vcoef_pitch(int nex) { return (nex + 3) & ~3; }
__host__ __device__ inline int64_t vcoef_index(int g, int ex, int ey, int ez, int pitch, int ney) {
  return (((int64_t)ez * 27 + g) * ney + ey) * pitch + ex;
}
__host__ __device__ inline int64_t vcoef_size(int nex, int ney, int nez) {
  return (int64_t)27 * nez * ney * vcoef_pitch(nex);
}

// Deterministic sum of one double per thread over a block (any 1-3D shape with a
// multiple of 32 threads): warp shuffle trees, then warp 0 sums the warp totals in
// order.  `scratch` is shared memory for >= 32 doubles; every thread must call
// (it contains a barrier); the result is valid in thread 0.
__device__ __forceinline__ double block_sum_dbl(double v, double* scratch) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nw = (blockDim.x * blockDim.y * blockDim.z) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((tid & 31) == 0) scratch[tid >> 5] = v;
  __syncthreads();
  double s = 0.;
  if (tid == 0)
    for (int w = 0; w < nw; w++) s += scratch[w];
  return s;
}

}  // namespace vfgpu
