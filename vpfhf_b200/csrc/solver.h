// solver.h -- vector kernels of the U/V solves (solver.cu).
#pragma once

#include "cg.cuh"

namespace vfgpu {

// out[q] = a[q] . b[q] for q < k (k <= 3); a, b are host arrays of device pointers.
cudaError_t dev_dots(const double* const* a, const double* const* b, int k, int64_t n,
                     double* partial, double* out, cudaStream_t s);
cudaError_t dev_znorm2(const double* r, const double* dinv, int64_t n, double* partial,
                       double* out, cudaStream_t s);
cudaError_t dev_absmax_diff(const double* a, const double* b, int64_t n, double* partial,
                            double* out, cudaStream_t s);
cudaError_t dev_u_residual(const double* y, const double* f, const double* u, const uint8_t* kind,
                           const double* bcu, double* F, int64_t n3, cudaStream_t s);
cudaError_t dev_apply_bc(double* u, const uint8_t* kind, const double* bcu, int64_t n,
                         cudaStream_t s);
cudaError_t dev_axpy(double* y, double a, const double* x, int64_t n, cudaStream_t s);
cudaError_t dev_axpby(double* z, const double* x, double a, const double* y, int64_t n,
                      cudaStream_t s);
cudaError_t dev_inv(const double* d, double* dinv, float* dinv32, int64_t n, cudaStream_t s);
cudaError_t dev_to_f32(const double* x, float* y, int64_t n, cudaStream_t s);
cudaError_t dev_add_f32(double* y, const float* x, int64_t n, cudaStream_t s);
cudaError_t dev_v_residual(const double* y, const double* b, const double* v, const double* virrev,
                           const uint8_t* kind, double irrevtol, int at2, double* F, int64_t n,
                           cudaStream_t s);
cudaError_t dev_vi_norm2(const double* F, const double* x, const double* lb, const double* ub,
                         int64_t n, double* partial, double* out, cudaStream_t s);
cudaError_t dev_v_mask(const double* F, const double* x, const double* lb, const double* ub,
                       const double* virrev, const uint8_t* kind, double irrevtol, int at2,
                       uint8_t* mask, int64_t n, cudaStream_t s);
cudaError_t dev_v_fix_step(double* Y, const double* F, const uint8_t* mask, const uint8_t* kind,
                           int64_t n, cudaStream_t s);
cudaError_t dev_v_project(const double* v, const double* Y, double lambda, const double* lb,
                          const double* ub, double* W, int64_t n, double* partial, double* out,
                          cudaStream_t s);
cudaError_t dev_v_bounds(const double* virrev, int at1, double* lb, double* ub, double* v,
                         int64_t n, cudaStream_t s);

}  // namespace vfgpu
