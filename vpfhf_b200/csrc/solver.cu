// solver.cu -- reductions, PCG kernels and the vector kernels of the U/V solves.
#include <cmath>

#include "cg.cuh"
#include "solver.h"

namespace vfgpu {

namespace {

// Block-level fixed-order tree sum of K values per thread into partial[blockIdx*K + q].
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* __restrict__ partial) {
  __shared__ double red[K][RED_THREADS];
#pragma unroll
  for (int q = 0; q < K; q++) red[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int st = RED_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
#pragma unroll
      for (int q = 0; q < K; q++) red[q][threadIdx.x] += red[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < K) partial[blockIdx.x * K + threadIdx.x] = red[threadIdx.x][0];
}

// Fixed-order sum of the per-block partials (one block).
template <int K>
__device__ __forceinline__ void final_sum(const double* __restrict__ partial, double (&out)[K]) {
  __shared__ double red[K][RED_THREADS];
  double v[K];
#pragma unroll
  for (int q = 0; q < K; q++) v[q] = 0.;
  for (int b = threadIdx.x; b < RED_BLOCKS; b += RED_THREADS)
#pragma unroll
    for (int q = 0; q < K; q++) v[q] += partial[b * K + q];
#pragma unroll
  for (int q = 0; q < K; q++) red[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int st = RED_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
#pragma unroll
      for (int q = 0; q < K; q++) red[q][threadIdx.x] += red[q][threadIdx.x + st];
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < K; q++) out[q] = red[q][0];
}

#define GRID_LOOP(i, n)                                                                  \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n);              \
       i += (int64_t)gridDim.x * blockDim.x)

// 16-byte packets for the bandwidth-bound CG kernels: W values of T per load/store.
// The CG vectors are whole cudaMalloc allocations (256-byte aligned); the n % W tail
// is done with scalar accesses by the first threads of the grid.
template <typename T> struct Pack {
  static constexpr int W = 16 / sizeof(T);
  T e[W];
};
template <typename T>
__device__ __forceinline__ Pack<T> ld16(const T* __restrict__ a, int64_t c) {
  Pack<T> p;
  if constexpr (sizeof(T) == 8) {
    const double2 q = reinterpret_cast<const double2*>(a)[c];
    p.e[0] = q.x;
    p.e[1] = q.y;
  } else {
    const float4 q = reinterpret_cast<const float4*>(a)[c];
    p.e[0] = q.x;
    p.e[1] = q.y;
    p.e[2] = q.z;
    p.e[3] = q.w;
  }
  return p;
}
template <typename T>
__device__ __forceinline__ void st16(T* __restrict__ a, int64_t c, const Pack<T>& p) {
  if constexpr (sizeof(T) == 8) {
    reinterpret_cast<double2*>(a)[c] = make_double2(p.e[0], p.e[1]);
  } else {
    reinterpret_cast<float4*>(a)[c] = make_float4(p.e[0], p.e[1], p.e[2], p.e[3]);
  }
}
// Visits the n values as 16-byte packets (fp(packet index)), then the tail of
// n % W values one by one (ft(element index)).
template <typename T, class FP, class FT>
__device__ __forceinline__ void pack_loop(int64_t n, FP fp, FT ft) {
  constexpr int W = Pack<T>::W;
  const int64_t np = n / W;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = t0; c < np; c += st) fp(c);
  for (int64_t i = np * W + t0; i < n; i += st) ft(i);
}
// The same packs visited from the end of the vectors back (for an elementwise kernel
// that follows a forward pass over some of the same vectors: it starts on the lines that
// pass left in L2).
template <typename T, class FP, class FT>
__device__ __forceinline__ void pack_loop_rev(int64_t n, FP fp, FT ft) {
  constexpr int W = Pack<T>::W;
  const int64_t np = n / W;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = np * W + t0; i < n; i += st) ft(i);
  for (int64_t c = t0; c < np; c += st) fp(np - 1 - c);
}

template <typename T>
__global__ void __launch_bounds__(RED_THREADS) cg_init_kernel(CGVecs<T> v, double* partial) {
  double acc[2] = {0., 0.};
  GRID_LOOP(i, v.n) {
    const bool m = v.mask && v.mask[i];
    const T r = m ? T(0) : v.b[i];
    const T z = r * v.dinv[i];
    v.x[i] = T(0);
    v.r[i] = r;
    v.p[i] = z;
    acc[0] += (double)z * (double)r;
    acc[1] += (double)z * (double)z;
  }
  block_sum<2>(acc, partial);
}

__global__ void cg_init_final(CGState* st, const double* partial, double rtol, double atol,
                              double dtol, int maxit) {
  double s[2];
  final_sum<2>(partial, s);
  if (threadIdx.x == 0) {
    st->rz = s[0];
    st->zz = s[1];
    st->rnorm0 = sqrt(s[1]);
    st->ttol = fmax(rtol * st->rnorm0, atol);
    st->dtol = dtol;
    st->its = 0;
    st->xalpha = 0.;
    st->maxit = maxit;
    st->arrive = 0;
    st->done = 0;
    st->reason = CG_RUNNING;
    if (!(st->rnorm0 == st->rnorm0)) {
      st->done = 1;
      st->reason = CG_DIVERGED_NAN;
    } else if (st->rnorm0 <= st->ttol) {
      st->done = 1;
      st->reason = st->rnorm0 <= atol ? CG_CONVERGED_ATOL : CG_CONVERGED_RTOL;
    } else if (s[0] == 0.) {
      st->done = 1;
      st->reason = CG_CONVERGED_ATOL;
    }
  }
}

// Fixed-order sum of n block partials by one block; every thread gets the result
// (identical in every block that calls it).  L1 is bypassed: the partials were
// written by other blocks or by an earlier kernel.
__device__ __forceinline__ double sum_partials(const double* __restrict__ p, int n) {
  __shared__ double red[RED_THREADS];
  double v = 0.;
  for (int b = threadIdx.x; b < n; b += RED_THREADS) v += __ldcg(p + b);
  red[threadIdx.x] = v;
  __syncthreads();
  for (int st = RED_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  const double s = red[0];
  __syncthreads();
  return s;
}

// End of a CG iteration from the new (r, z) and (z, z): iteration count,
// convergence tests (KSPConvergedDefault on the preconditioned norm) and beta.
__device__ __forceinline__ void cg_finish_iteration(CGState* st, double rz, double zz) {
  st->its += 1;
  st->zz = zz;
  const double dp = sqrt(zz);
  if (!(dp == dp)) {
    st->done = 1;
    st->reason = CG_DIVERGED_NAN;
  } else if (dp <= st->ttol) {
    st->done = 1;
    st->reason = CG_CONVERGED_RTOL;
  } else if (dp >= st->dtol * st->rnorm0) {
    st->done = 1;
    st->reason = CG_DIVERGED_DTOL;
  } else if (st->its >= st->maxit) {
    st->done = 1;
    st->reason = CG_DIVERGED_ITS;
  } else {
    st->beta = rz / st->rz;
    st->rz = rz;
    if (rz == 0.) {
      st->done = 1;
      st->reason = CG_CONVERGED_ATOL;
    }
  }
}

// p.w by blocks (for an operator apply that did not produce it).
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) cg_pw_kernel(CGVecs<T> v, const CGState* st,
                                                            double* partial) {
  if (st->done) return;
  double acc[1] = {0.};
  pack_loop<T>(
      v.n,
      [&](int64_t c) {
        const Pack<T> p = ld16(v.p, c), w = ld16(v.w, c);
#pragma unroll
        for (int k = 0; k < Pack<T>::W; k++) acc[0] += (double)p.e[k] * (double)w.e[k];
      },
      [&](int64_t i) { acc[0] += (double)v.p[i] * (double)v.w[i]; });
  block_sum<1>(acc, partial);
}

// One CG step after w = A p: every block sums the operator's p.w partials (written
// by the tile and seam kernels of the apply) to the same alpha = (r,z)/(p,w), updates
// x and r, and adds its share of (r,z), (z,z) with z = D^-1 r; the last block to
// finish sums those partials and ends the iteration (cg_finish_iteration).  The
// arrival counter is the only atomic; every sum has a fixed order.
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) cg_update_kernel(CGVecs<T> v, CGState* st,
                                                                double* partial) {
  if (st->done) return;
  const double pw = sum_partials(v.dotp, v.ndot);
  if (!(pw > 0.)) {  // same value in every block: all of them stop here
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->pw = pw;
      st->xalpha = 0.;  // no step of this iteration reaches x
      st->done = 1;
      st->reason = (pw == pw) ? CG_DIVERGED_INDEFINITE : CG_DIVERGED_NAN;
    }
    return;
  }
  const double alpha = st->rz / pw;  // st->rz changes only after every block has arrived
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->pw = pw;
    st->alpha = alpha;
    st->xalpha = alpha;  // x += alpha p: in cg_p_kernel, or in cg_finish_x if the solve stops here
  }
  const T a = (T)alpha;
  double acc[2] = {0., 0.};
  pack_loop<T>(
      v.n,
      [&](int64_t c) {
        Pack<T> r = ld16(v.r, c);
        const Pack<T> w = ld16(v.w, c), d = ld16(v.dinv, c);
#pragma unroll
        for (int k = 0; k < Pack<T>::W; k++) {
          r.e[k] = r.e[k] - a * w.e[k];
          const T z = r.e[k] * d.e[k];
          acc[0] += (double)z * (double)r.e[k];
          acc[1] += (double)z * (double)z;
        }
        st16(v.r, c, r);
      },
      [&](int64_t i) {
        const T r = v.r[i] - a * v.w[i];
        const T z = r * v.dinv[i];
        v.r[i] = r;
        acc[0] += (double)z * (double)r;
        acc[1] += (double)z * (double)z;
      });
  block_sum<2>(acc, partial);
  __shared__ bool last;
  __threadfence();  // this block's partials are visible before it is counted
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->arrive, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double sum[2] = {0., 0.};
  {
    __shared__ double red[2][RED_THREADS];
    for (int b = threadIdx.x; b < (int)gridDim.x; b += RED_THREADS) {
      sum[0] += __ldcg(partial + 2 * b);
      sum[1] += __ldcg(partial + 2 * b + 1);
    }
    red[0][threadIdx.x] = sum[0];
    red[1][threadIdx.x] = sum[1];
    __syncthreads();
    for (int s2 = RED_THREADS / 2; s2 > 0; s2 >>= 1) {
      if (threadIdx.x < s2) {
        red[0][threadIdx.x] += red[0][threadIdx.x + s2];
        red[1][threadIdx.x] += red[1][threadIdx.x + s2];
      }
      __syncthreads();
    }
    sum[0] = red[0][0];
    sum[1] = red[1][0];
  }
  if (threadIdx.x == 0) {
    st->arrive = 0;
    cg_finish_iteration(st, sum[0], sum[1]);
  }
}

// x += alpha p and p = z + beta p in one pass (the iteration went on: not done),
// back from the end of the vectors: the update kernel's forward pass left the tail of r
// and dinv in L2.
template <typename T>
__global__ void cg_p_kernel(CGVecs<T> v, const CGState* st) {
  if (st->done) return;
  const T a = (T)st->alpha, b = (T)st->beta;
  pack_loop_rev<T>(
      v.n,
      [&](int64_t c) {
        Pack<T> p = ld16(v.p, c), x = ld16(v.x, c);
        const Pack<T> r = ld16(v.r, c), d = ld16(v.dinv, c);
#pragma unroll
        for (int k = 0; k < Pack<T>::W; k++) {
          x.e[k] = x.e[k] + a * p.e[k];
          p.e[k] = r.e[k] * d.e[k] + b * p.e[k];
        }
        st16(v.x, c, x);
        st16(v.p, c, p);
      },
      [&](int64_t i) {
        v.x[i] = v.x[i] + a * v.p[i];
        v.p[i] = v.r[i] * v.dinv[i] + b * v.p[i];
      });
}

// The step of the iteration that stopped the solve (its cg_p_kernel did not run):
// x += xalpha p; nothing after an indefinite p.w (xalpha = 0) or while the solve is
// still going (a watchdog stop between iterations: every step has reached x).
template <typename T>
__global__ void cg_finish_x_kernel(CGVecs<T> v, const CGState* st) {
  if (!st->done) return;
  const double alpha = st->xalpha;
  if (alpha == 0.) return;
  const T a = (T)alpha;
  pack_loop<T>(
      v.n,
      [&](int64_t c) {
        Pack<T> x = ld16(v.x, c);
        const Pack<T> p = ld16(v.p, c);
#pragma unroll
        for (int k = 0; k < Pack<T>::W; k++) x.e[k] = x.e[k] + a * p.e[k];
        st16(v.x, c, x);
      },
      [&](int64_t i) { v.x[i] = v.x[i] + a * v.p[i]; });
}

// ---- generic vector kernels ----
template <int K> struct PtrPack {
  const double* p[K];
};

template <int K>
__global__ void __launch_bounds__(RED_THREADS) dots_kernel(PtrPack<K> a, PtrPack<K> b, int64_t n,
                                                           double* partial) {
  double acc[K];
#pragma unroll
  for (int q = 0; q < K; q++) acc[q] = 0.;
  GRID_LOOP(i, n) {
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] += a.p[q][i] * b.p[q][i];
  }
  block_sum<K>(acc, partial);
}

template <int K>
__global__ void dots_final(const double* partial, double* out) {
  double s[K];
  final_sum<K>(partial, s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < K; q++) out[q] = s[q];
}

__global__ void __launch_bounds__(RED_THREADS) absmax_diff_kernel(const double* a, const double* b,
                                                                  int64_t n, double* partial) {
  __shared__ double red[RED_THREADS];
  double m = 0.;
  GRID_LOOP(i, n) m = fmax(m, fabs(a[i] - b[i]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int st = RED_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void absmax_final(const double* partial, double* out) {
  if (threadIdx.x == 0) {
    double m = 0.;
    for (int b = 0; b < RED_BLOCKS; b++) m = fmax(m, partial[b]);
    out[0] = m;
  }
}

// F = y - f on free dofs, F = u - ubc on Dirichlet dofs (ResidualApplyDirichletBC).
__global__ void u_residual_kernel(const double* y, const double* f, const double* u,
                                  const uint8_t* kind, const double* bcu, double* F, int64_t n3) {
  GRID_LOOP(i, n3) {
    const int k = kind ? kind[i] : 0;
    if (k == 0)
      F[i] = y[i] - f[i];
    else
      F[i] = u[i] - (k == 1 ? 0. : k == 2 ? 1. : bcu[i]);
  }
}

// U := Dirichlet value on Dirichlet dofs (VecApplyDirichletBC).
__global__ void apply_bc_kernel(double* u, const uint8_t* kind, const double* bcu, int64_t n) {
  GRID_LOOP(i, n) {
    const int k = kind[i];
    if (k) u[i] = k == 1 ? 0. : k == 2 ? 1. : (bcu ? bcu[i] : u[i]);
  }
}

__global__ void axpy_kernel(double* y, double a, const double* x, int64_t n) {
  GRID_LOOP(i, n) y[i] += a * x[i];
}
__global__ void axpby_kernel(double* z, const double* x, double a, const double* y, int64_t n) {
  GRID_LOOP(i, n) z[i] = x[i] + a * y[i];
}
__global__ void inv_kernel(const double* d, double* dinv, float* dinv32, int64_t n) {
  GRID_LOOP(i, n) {
    const double r = 1. / d[i];
    dinv[i] = r;
    if (dinv32) dinv32[i] = (float)r;
  }
}
__global__ void to_f32_kernel(const double* x, float* y, int64_t n) {
  GRID_LOOP(i, n) y[i] = (float)x[i];
}
__global__ void add_f32_kernel(double* y, const float* x, int64_t n) {
  GRID_LOOP(i, n) y[i] += (double)x[i];
}

// ---- V (phase field) ----
// F_V = y - b; AT2 irreversibility rows 0 (VF_IrrevApplyEQVec); BC rows v - bc.
__global__ void v_residual_kernel(const double* y, const double* b, const double* v,
                                  const double* virrev, const uint8_t* kind, double irrevtol,
                                  int at2, double* F, int64_t n) {
  GRID_LOOP(i, n) {
    double f = y[i] - b[i];
    if (at2 && virrev[i] <= irrevtol) f = 0.;
    const int k = kind ? kind[i] : 0;
    if (k) f = v[i] - (k == 1 ? 0. : k == 2 ? 1. : v[i]);
    F[i] = f;
  }
}

// VI norm (SNESVIComputeInactiveSetFnorm) partial sums.
__global__ void __launch_bounds__(RED_THREADS) vi_norm_kernel(const double* F, const double* x,
                                                              const double* lb, const double* ub,
                                                              int64_t n, double* partial) {
  double acc[1] = {0.};
  GRID_LOOP(i, n) {
    const double f = F[i];
    if ((x[i] > lb[i] + 1.e-8 || f <= 0.) && (x[i] < ub[i] - 1.e-8 || f >= 0.)) acc[0] += f * f;
  }
  block_sum<1>(acc, partial);
}

// Active set of SNESVINEWTONRSLS (x at a bound with F pushing outward) plus the
// dofs removed from the reduced system (Dirichlet rows, AT2 irreversibility).
__global__ void v_mask_kernel(const double* F, const double* x, const double* lb, const double* ub,
                              const double* virrev, const uint8_t* kind, double irrevtol, int at2,
                              uint8_t* mask, int64_t n) {
  GRID_LOOP(i, n) {
    const double f = F[i];
    const bool inactive = (x[i] > lb[i] + 1.e-8 || f < 0.) && (x[i] < ub[i] - 1.e-8 || f > 0.);
    const bool fixed = (kind && kind[i]) || (at2 && virrev[i] <= irrevtol);
    mask[i] = (!inactive || fixed) ? 1 : 0;
  }
}

// Newton step on the removed dofs: Dirichlet rows are identity (Y = F), active
// and irreversible dofs do not move.
__global__ void v_fix_step_kernel(double* Y, const double* F, const uint8_t* mask,
                                  const uint8_t* kind, int64_t n) {
  GRID_LOOP(i, n) {
    if (mask[i]) Y[i] = (kind && kind[i]) ? F[i] : 0.;
  }
}

// W = clamp(v - lambda Y, lb, ub) (SNESVIProjectOntoBounds), and partial |W - v|^2.
__global__ void __launch_bounds__(RED_THREADS) v_project_kernel(const double* v, const double* Y,
                                                                double lambda, const double* lb,
                                                                const double* ub, double* W,
                                                                int64_t n, double* partial) {
  double acc[1] = {0.};
  GRID_LOOP(i, n) {
    const double w = fmin(fmax(v[i] - lambda * Y[i], lb[i]), ub[i]);
    W[i] = w;
    acc[0] += (w - v[i]) * (w - v[i]);
  }
  block_sum<1>(acc, partial);
}

__global__ void v_bounds_kernel(const double* virrev, int at1, double* lb, double* ub, double* v,
                                int64_t n) {
  GRID_LOOP(i, n) {
    const double l = 0., u = at1 ? virrev[i] : 1.;
    lb[i] = l;
    ub[i] = u;
    v[i] = fmin(fmax(v[i], l), u);
  }
}

inline int vgrid(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

}  // namespace

// ------------------------------------------------------------------ host wrappers
template <typename T>
cudaError_t cg_init(const CGVecs<T>& v, CGState* st, double* partial, double rtol, double atol,
                    double dtol, int maxit, cudaStream_t s) {
  cg_init_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(v, partial);
  cg_init_final<<<1, RED_THREADS, 0, s>>>(st, partial, rtol, atol, dtol, maxit);
  return cudaGetLastError();
}

template <typename T> static bool aligned16(const CGVecs<T>& v) {
  const void* ps[] = {v.x, v.r, v.p, v.w, v.dinv};
  for (const void* p : ps)
    if (reinterpret_cast<uintptr_t>(p) % 16) return false;
  return true;
}

template <typename T>
cudaError_t cg_after_apply(const CGVecs<T>& v, CGState* st, double* partial, cudaStream_t s) {
  if (!aligned16(v)) return cudaErrorMisalignedAddress;  // caught on the host, nothing launched
  if (!v.dotp) {  // the apply did not accumulate p.w: a separate pass into partial[2R, 3R)
    cg_pw_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(v, st, partial + 2 * RED_BLOCKS);
    CGVecs<T> u = v;
    u.dotp = partial + 2 * RED_BLOCKS;
    u.ndot = RED_BLOCKS;
    cg_update_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(u, st, partial);
  } else {
    if (v.ndot <= 0) return cudaErrorInvalidValue;
    cg_update_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(v, st, partial);
  }
  cg_p_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(v, st);
  return cudaGetLastError();
}

template <typename T>
cudaError_t cg_finish_x(const CGVecs<T>& v, const CGState* st, cudaStream_t s) {
  if (!aligned16(v)) return cudaErrorMisalignedAddress;
  cg_finish_x_kernel<T><<<RED_BLOCKS, RED_THREADS, 0, s>>>(v, st);
  return cudaGetLastError();
}

template cudaError_t cg_init<double>(const CGVecs<double>&, CGState*, double*, double, double,
                                     double, int, cudaStream_t);
template cudaError_t cg_init<float>(const CGVecs<float>&, CGState*, double*, double, double,
                                    double, int, cudaStream_t);
template cudaError_t cg_after_apply<double>(const CGVecs<double>&, CGState*, double*,
                                            cudaStream_t);
template cudaError_t cg_after_apply<float>(const CGVecs<float>&, CGState*, double*, cudaStream_t);
template cudaError_t cg_finish_x<double>(const CGVecs<double>&, const CGState*, cudaStream_t);
template cudaError_t cg_finish_x<float>(const CGVecs<float>&, const CGState*, cudaStream_t);

template <int K>
static void launch_dots(const double* const* a, const double* const* b, int64_t n, double* partial,
                        double* out, cudaStream_t s) {
  PtrPack<K> pa, pb;
  for (int q = 0; q < K; q++) {
    pa.p[q] = a[q];
    pb.p[q] = b[q];
  }
  dots_kernel<K><<<RED_BLOCKS, RED_THREADS, 0, s>>>(pa, pb, n, partial);
  dots_final<K><<<1, RED_THREADS, 0, s>>>(partial, out);
}

cudaError_t dev_dots(const double* const* a, const double* const* b, int k, int64_t n,
                     double* partial, double* out, cudaStream_t s) {
  // a, b: host arrays of k device pointers; out[q] = a[q] . b[q] (device memory)
  switch (k) {
    case 1: launch_dots<1>(a, b, n, partial, out, s); break;
    case 2: launch_dots<2>(a, b, n, partial, out, s); break;
    case 3: launch_dots<3>(a, b, n, partial, out, s); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

namespace {
__global__ void __launch_bounds__(RED_THREADS) znorm_kernel(const double* r, const double* dinv,
                                                            int64_t n, double* partial) {
  double acc[1] = {0.};
  GRID_LOOP(i, n) {
    const double z = r[i] * dinv[i];
    acc[0] += z * z;
  }
  block_sum<1>(acc, partial);
}
}  // namespace

cudaError_t dev_znorm2(const double* r, const double* dinv, int64_t n, double* partial,
                       double* out, cudaStream_t s) {
  znorm_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(r, dinv, n, partial);
  dots_final<1><<<1, RED_THREADS, 0, s>>>(partial, out);
  return cudaGetLastError();
}

cudaError_t dev_absmax_diff(const double* a, const double* b, int64_t n, double* partial,
                            double* out, cudaStream_t s) {
  absmax_diff_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a, b, n, partial);
  absmax_final<<<1, 32, 0, s>>>(partial, out);
  return cudaGetLastError();
}

cudaError_t dev_u_residual(const double* y, const double* f, const double* u, const uint8_t* kind,
                           const double* bcu, double* F, int64_t n3, cudaStream_t s) {
  u_residual_kernel<<<vgrid(n3), 256, 0, s>>>(y, f, u, kind, bcu, F, n3);
  return cudaGetLastError();
}
cudaError_t dev_apply_bc(double* u, const uint8_t* kind, const double* bcu, int64_t n,
                         cudaStream_t s) {
  apply_bc_kernel<<<vgrid(n), 256, 0, s>>>(u, kind, bcu, n);
  return cudaGetLastError();
}
cudaError_t dev_axpy(double* y, double a, const double* x, int64_t n, cudaStream_t s) {
  axpy_kernel<<<vgrid(n), 256, 0, s>>>(y, a, x, n);
  return cudaGetLastError();
}
cudaError_t dev_axpby(double* z, const double* x, double a, const double* y, int64_t n,
                      cudaStream_t s) {
  axpby_kernel<<<vgrid(n), 256, 0, s>>>(z, x, a, y, n);
  return cudaGetLastError();
}
cudaError_t dev_inv(const double* d, double* dinv, float* dinv32, int64_t n, cudaStream_t s) {
  inv_kernel<<<vgrid(n), 256, 0, s>>>(d, dinv, dinv32, n);
  return cudaGetLastError();
}
cudaError_t dev_to_f32(const double* x, float* y, int64_t n, cudaStream_t s) {
  to_f32_kernel<<<vgrid(n), 256, 0, s>>>(x, y, n);
  return cudaGetLastError();
}
cudaError_t dev_add_f32(double* y, const float* x, int64_t n, cudaStream_t s) {
  add_f32_kernel<<<vgrid(n), 256, 0, s>>>(y, x, n);
  return cudaGetLastError();
}
cudaError_t dev_v_residual(const double* y, const double* b, const double* v, const double* virrev,
                           const uint8_t* kind, double irrevtol, int at2, double* F, int64_t n,
                           cudaStream_t s) {
  v_residual_kernel<<<vgrid(n), 256, 0, s>>>(y, b, v, virrev, kind, irrevtol, at2, F, n);
  return cudaGetLastError();
}
cudaError_t dev_vi_norm2(const double* F, const double* x, const double* lb, const double* ub,
                         int64_t n, double* partial, double* out, cudaStream_t s) {
  vi_norm_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(F, x, lb, ub, n, partial);
  dots_final<1><<<1, RED_THREADS, 0, s>>>(partial, out);
  return cudaGetLastError();
}
cudaError_t dev_v_mask(const double* F, const double* x, const double* lb, const double* ub,
                       const double* virrev, const uint8_t* kind, double irrevtol, int at2,
                       uint8_t* mask, int64_t n, cudaStream_t s) {
  v_mask_kernel<<<vgrid(n), 256, 0, s>>>(F, x, lb, ub, virrev, kind, irrevtol, at2, mask, n);
  return cudaGetLastError();
}
cudaError_t dev_v_fix_step(double* Y, const double* F, const uint8_t* mask, const uint8_t* kind,
                           int64_t n, cudaStream_t s) {
  v_fix_step_kernel<<<vgrid(n), 256, 0, s>>>(Y, F, mask, kind, n);
  return cudaGetLastError();
}
cudaError_t dev_v_project(const double* v, const double* Y, double lambda, const double* lb,
                          const double* ub, double* W, int64_t n, double* partial, double* out,
                          cudaStream_t s) {
  v_project_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(v, Y, lambda, lb, ub, W, n, partial);
  dots_final<1><<<1, RED_THREADS, 0, s>>>(partial, out);
  return cudaGetLastError();
}
cudaError_t dev_v_bounds(const double* virrev, int at1, double* lb, double* ub, double* v,
                         int64_t n, cudaStream_t s) {
  v_bounds_kernel<<<vgrid(n), 256, 0, s>>>(virrev, at1, lb, ub, v, n);
  return cudaGetLastError();
}

}  // namespace vfgpu
