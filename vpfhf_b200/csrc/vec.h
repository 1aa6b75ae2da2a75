// vec.h -- elementwise helper launchers.
#pragma once

#include <algorithm>

#include "common.cuh"

namespace vfgpu {
cudaError_t convert_f64_f32(const double* x, float* y, int64_t n, cudaStream_t s);
cudaError_t convert_f32_f64(const float* x, double* y, int64_t n, cudaStream_t s);
cudaError_t fill_f64(double* x, double a, int64_t n, cudaStream_t s);
}  // namespace vfgpu
