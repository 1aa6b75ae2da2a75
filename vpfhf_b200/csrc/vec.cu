// vec.cu -- elementwise helpers (precision conversion, fills).
#include "vec.h"

namespace vfgpu {

namespace {
template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ x, B* __restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (B)x[i];
}
__global__ void fill_kernel(double* __restrict__ x, double a, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = a;
}
inline int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }
}  // namespace

cudaError_t convert_f64_f32(const double* x, float* y, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  convert_kernel<double, float><<<grid_for(n), 256, 0, s>>>(x, y, n);
  return cudaGetLastError();
}
cudaError_t convert_f32_f64(const float* x, double* y, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  convert_kernel<float, double><<<grid_for(n), 256, 0, s>>>(x, y, n);
  return cudaGetLastError();
}
cudaError_t fill_f64(double* x, double a, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  fill_kernel<<<grid_for(n), 256, 0, s>>>(x, a, n);
  return cudaGetLastError();
}

}  // namespace vfgpu
