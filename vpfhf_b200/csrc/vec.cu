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

namespace {
// 16 independent FMA chains per thread; values stay bounded (|a| < 1).
template <typename T>
__global__ void fma_peak_kernel(T* out, int iters, T a, T b) {
  T x[16];
#pragma unroll
  for (int q = 0; q < 16; q++) x[q] = T(threadIdx.x + q) * T(1e-7);
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int q = 0; q < 16; q++) x[q] = fma(x[q], a, b);
  T s = T(0);
#pragma unroll
  for (int q = 0; q < 16; q++) s += x[q];
  if (s == T(12345.678)) out[0] = s;  // keeps the chains alive
}
}  // namespace

template <typename T>
static double fma_peak(int nsm) {
  T* out = nullptr;
  if (cudaMalloc((void**)&out, sizeof(T)) != cudaSuccess) return -1;
  const int threads = 256, blocks = nsm * 8, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_peak_kernel<T><<<blocks, threads>>>(out, iters / 8, T(0.999999), T(1e-7));  // warm-up
  cudaEventRecord(e0);
  fma_peak_kernel<T><<<blocks, threads>>>(out, iters, T(0.999999), T(1e-7));
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0) return -1;
  return 2.0 * 16.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e12;
}

double fma_peak_tflops(int bytes, int nsm) {
  return bytes == 8 ? fma_peak<double>(nsm) : fma_peak<float>(nsm);
}

}  // namespace vfgpu

extern "C" int vfgpu_fma_peak(int bytes, double* tflops) {
  if (!tflops || (bytes != 4 && bytes != 8)) return -1;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const double t = vfgpu::fma_peak_tflops(bytes, nsm);
  if (t <= 0) return -2;
  *tflops = t;
  return 0;
}
