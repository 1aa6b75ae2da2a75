// mg.cu -- geometric multigrid V-cycle as the preconditioner of the U solve's CG
// (solve option VFGPU_PC_MG).  No counterpart in the reference, whose snesU uses
// KSPCG with Jacobi (or hypre when PETSc has it, VFCommon.c:1044-1047); the solve it
// feeds keeps the reference's semantics (same residual, same SNES tests, the CG
// stopping test of the Jacobi solve), only the Krylov iterations get fewer.
//
// Each coarser level has ceil(cells / 2) uniform cells along every axis that still has
// >= 9 nodes (the others keep theirs), over the same box: nested where a cell count is
// even, offset by a fraction of a cell where it is odd.  Each coarse level
// rediscretises the same operator (the tile engine's U apply) on its grid with the
// phase field interpolated at its nodes (nested: v_c(I) = v_f(2I)), the Dirichlet
// bits of the nearest fine node, the element layer of the lowest fine layer it holds
// and, for a per-cell modulus, the mean of the fine cells whose centres it holds
// (nested: the 8 children).  Transfers: trilinear prolongation and its exact
// transpose, Dirichlet dofs excluded on both sides.  Smoother: Chebyshev
// iteration of D^-1 K (degree kSmoothDeg) on [lmax/10, lmax] (lmax = 1.1 x the
// estimate of 12 power iterations per level, 4 from the previous vector once there is
// one), pre and post; the coarsest level runs degree kCoarseDeg on [lmax/100, lmax].  Every step is a fixed sequence of
// deterministic kernels reading its Chebyshev coefficients from device memory, so
// the V-cycle is a fixed symmetric linear operator (plain PCG applies) and is
// replayed as one CUDA graph.
//
// Precision: the V-cycle runs in FP64 (solve precision FP64) or FP32 (MIXED); the
// outer CG, its residual and its stopping test stay FP64 in both.
#include <algorithm>
#include <cmath>
#include <functional>
#include <vector>

#include "abi_util.h"
#include "ops.cuh"
#include "solver.h"
#include "vec.h"

namespace vfgpu {
namespace {

// Power iterations per level: from the deterministic seed at the first set-up, then
// from the previous set-up's vector (the operator of the next StepU differs by the
// phase field's update only).
// Degrees: measured on B200 (StepU, 129^3 and 257^3 penny cracks, c5 set-up at 129^3
// and 193^3), degree 1 pre and post smoothing with a 15-step coarsest solve beat the
// higher degrees on time although the CG takes more iterations (257^3: 0.163 s mixed
// with 20 iterations against 0.181 s / 15 for degree 2 and 0.209 s / 13 for degree 3).
// 2 warm power iterations instead of 4 cost one more CG iteration per StepU in the
// 129^3 AM loop (4 AM steps: 87.3 against 85.9 ms mixed).
constexpr int kSmoothDeg = 1, kCoarseDeg = 15, kPowerIts = 12, kWarmPowerIts = 4;
constexpr double kSmoothLo = 0.1, kCoarseLo = 0.01, kLmaxSafety = 1.1;
constexpr int kCoefPerLevel = 64;  // [0] lmax [1] 1/theta [2..59] (c1, c2) [62..63] scratch
constexpr int kPowBlocks = 296, kPowThreads = 256;
constexpr int kGraphMG64 = 5, kGraphMG32 = 6;  // vfgpu_ctx::Graph kinds

inline int blocks_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

#define GRID_STRIDE(i, n)                                                                \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n);              \
       i += (int64_t)gridDim.x * blockDim.x)

// Grid transfers between a level and the next coarser one.  Along each axis the coarse
// grid spans the same interval with nc nodes (nc - 1 = ceil((nf - 1) / 2) cells, or
// nc = nf on an axis that is not coarsened), so fine node i sits at coarse coordinate
// i (nc - 1) / (nf - 1): in coarse cell I = floor of it with the linear weights
// (1 - w, w), w the fractional part, computed exactly from integers.  With an even
// fine cell count this is the nested case (w = 0 or 1/2 at the fine nodes 2I, 2I + 1).
struct Lin {
  int I;
  double whi;
};
__host__ __device__ __forceinline__ Lin fine_in_coarse(int i, int nf, int nc) {
  const long long num = (long long)i * (nc - 1), den = nf - 1;
  Lin l;
  l.I = (int)(num / den);
  l.whi = (double)(num - (long long)l.I * den) / (double)den;
  return l;
}

// One axis of the transfer between a level and the next coarser one, tabulated at the
// hierarchy's build: fine node i lies in coarse cell pI[i] with upper weight pw[i]
// (fine_in_coarse), and coarse node I's hat function covers the fine nodes
// [rlo[I], rlo[I] + rn[I]) (<= 4 for the ratios ceil(cells / 2) gives: the open
// interval of two coarse cells holds at most 4 fine nodes) with nonzero weight.
// Two common axes need no table (mode): a nested axis (an even fine cell count, ratio
// 2: fine node i in coarse cell i / 2 with upper weight 1/2 for odd i, coarse node I
// covering 2I - 1 .. 2I + 1) and an axis that is not coarsened (identity); both give
// the table's values exactly.
constexpr int kXferTable = 0, kXferNested = 1, kXferIdentity = 2;
struct XferAxis {
  const int* pI;
  const double* pw;
  const int* rlo;
  const int* rn;
  int nf, mode;
};
struct Xfer {
  XferAxis a[3];
};

// Weight of coarse node I at fine node i of its support (the prolongation's entry).
__device__ __forceinline__ double hat(const XferAxis& A, int i, int I) {
  if (A.mode == kXferNested) return i == 2 * I ? 1.0 : 0.5;
  if (A.mode == kXferIdentity) return 1.0;
  const double w = A.pw[i];
  return A.pI[i] == I ? 1.0 - w : w;
}
// The support [lo, lo + n) of coarse node I.
__device__ __forceinline__ void support_of(const XferAxis& A, int I, int& lo, int& n) {
  if (A.mode == kXferNested) {
    lo = max(2 * I - 1, 0);
    n = min(2 * I + 1, A.nf - 1) - lo + 1;
  } else if (A.mode == kXferIdentity) {
    lo = I;
    n = 1;
  } else {
    lo = A.rlo[I];
    n = A.rn[I];
  }
}
// The coarse cell of fine node i and its upper weight.
__device__ __forceinline__ void cell_of(const XferAxis& A, int i, int& I, double& whi) {
  if (A.mode == kXferNested) {
    I = i >> 1;
    whi = (i & 1) ? 0.5 : 0.0;
  } else if (A.mode == kXferIdentity) {
    I = i;
    whi = 0.0;
  } else {
    I = A.pI[i];
    whi = A.pw[i];
  }
}

// Restriction of the residual b - t (the transpose of prolong_add_kernel): coarse node I
// gathers the fine nodes of its hat function's support with the same weights, skipping
// fine Dirichlet dofs; coarse Dirichlet dofs are zeroed.
template <typename T>
__global__ void restrict_kernel(const T* __restrict__ bf, const T* __restrict__ tf,
                                const uint8_t* __restrict__ bc_f, int fx, int fy, const Xfer X,
                                T* __restrict__ rc, int cx, int cy, int cz,
                                const uint8_t* __restrict__ bc_c) {
  const int64_t Nc = (int64_t)cx * cy * cz;
  GRID_STRIDE(q, Nc) {
    const int I = (int)(q % cx), J = (int)((q / cx) % cy), K = (int)(q / ((int64_t)cx * cy));
    int x0, nxs, y0, nys, z0, nzs;
    support_of(X.a[0], I, x0, nxs);
    support_of(X.a[1], J, y0, nys);
    support_of(X.a[2], K, z0, nzs);
    double wx[4];
#pragma unroll
    for (int c1 = 0; c1 < 4; c1++) wx[c1] = c1 < nxs ? hat(X.a[0], x0 + c1, I) : 0.0;
    T acc[3] = {T(0), T(0), T(0)};
    // fully unrolled (predicated) so that the row loads of the support issue together
#pragma unroll
    for (int c3 = 0; c3 < 4; c3++) {
      if (c3 >= nzs) continue;
      const double wz = hat(X.a[2], z0 + c3, K);
#pragma unroll
      for (int c2 = 0; c2 < 4; c2++) {
        if (c2 >= nys) continue;
        const double wzy = wz * hat(X.a[1], y0 + c2, J);
        const int64_t row = node_index(x0, y0 + c2, z0 + c3, fx, fy);
#pragma unroll
        for (int c1 = 0; c1 < 4; c1++) {
          if (c1 < nxs) {
            const T w = T(wzy * wx[c1]);
            const int64_t n = row + c1;
            const unsigned bf_bits = bc_f[n];
#pragma unroll
            for (int c = 0; c < 3; c++)
              if (!((bf_bits >> c) & 1u)) acc[c] += w * (bf[3 * n + c] - tf[3 * n + c]);
          }
        }
      }
    }
    const unsigned b = bc_c[q];
    for (int c = 0; c < 3; c++) rc[3 * q + c] = ((b >> c) & 1u) ? T(0) : acc[c];
  }
}

// x_f += trilinear interpolation of e_c; fine Dirichlet dofs untouched.
template <typename T>
__global__ void prolong_add_kernel(const T* __restrict__ ec, int cx, int cy, const Xfer X,
                                   T* __restrict__ xf, int fx, int fy, int fz,
                                   const uint8_t* __restrict__ bc_f) {
  const int64_t Nf = (int64_t)fx * fy * fz;
  GRID_STRIDE(q, Nf) {
    const int i = (int)(q % fx), j = (int)((q / fx) % fy), k = (int)(q / ((int64_t)fx * fy));
    int Ix, Iy, Iz;
    double hx, hy, hz;
    cell_of(X.a[0], i, Ix, hx);
    cell_of(X.a[1], j, Iy, hy);
    cell_of(X.a[2], k, Iz, hz);
    T acc[3] = {T(0), T(0), T(0)};
    for (int dk = 0; dk < 2; dk++) {
      const double wzk = dk ? hz : 1.0 - hz;
      if (wzk == 0.0) continue;
      for (int dj = 0; dj < 2; dj++) {
        const double wyj = dj ? hy : 1.0 - hy;
        if (wyj == 0.0) continue;
        for (int di = 0; di < 2; di++) {
          const double wxi = di ? hx : 1.0 - hx;
          if (wxi == 0.0) continue;
          const T w = T(wzk * wyj * wxi);
          const int64_t n = node_index(Ix + di, Iy + dj, Iz + dk, cx, cy);
          for (int c = 0; c < 3; c++) acc[c] += w * ec[3 * n + c];
        }
      }
    }
    const unsigned b = bc_f[q];
    for (int c = 0; c < 3; c++)
      if (!((b >> c) & 1u)) xf[3 * q + c] += acc[c];
  }
}

// Coarse node I takes v interpolated at its position (in the nested case: fine node 2I)
// and the Dirichlet bits of the nearest fine node (box faces map to box faces).
__global__ void inject_kernel(const double* __restrict__ vf, const uint8_t* __restrict__ bcf,
                              int fx, int fy, int fz, double* __restrict__ vc,
                              uint8_t* __restrict__ bcc, int cx, int cy, int cz) {
  const int64_t Nc = (int64_t)cx * cy * cz;
  GRID_STRIDE(q, Nc) {
    const int I = (int)(q % cx), J = (int)((q / cx) % cy), K = (int)(q / ((int64_t)cx * cy));
    // coarse node in the fine grid's index space: fine_in_coarse with the roles swapped
    const Lin lx = fine_in_coarse(I, cx, fx), ly = fine_in_coarse(J, cy, fy),
              lz = fine_in_coarse(K, cz, fz);
    double v = 0.;
    for (int dk = 0; dk < 2; dk++) {
      const double wzk = dk ? lz.whi : 1.0 - lz.whi;
      if (wzk == 0.0) continue;
      for (int dj = 0; dj < 2; dj++) {
        const double wyj = dj ? ly.whi : 1.0 - ly.whi;
        if (wyj == 0.0) continue;
        for (int di = 0; di < 2; di++) {
          const double wxi = di ? lx.whi : 1.0 - lx.whi;
          if (wxi == 0.0) continue;
          v += wzk * wyj * wxi * vf[node_index(lx.I + di, ly.I + dj, lz.I + dk, fx, fy)];
        }
      }
    }
    vc[q] = v;
    const int ni = lx.I + (lx.whi > 0.5 ? 1 : 0), nj = ly.I + (ly.whi > 0.5 ? 1 : 0),
              nk = lz.I + (lz.whi > 0.5 ? 1 : 0);
    bcc[q] = bcf[node_index(ni, nj, nk, fx, fy)];
  }
}

// The fine cells (along one axis) whose centres lie in coarse cell k: [first, last).
__device__ __forceinline__ void fine_cells_of(int k, int ncf, int ncc, int& first, int& last) {
  // centre of fine cell j at coarse coordinate (j + 1/2) ncc / ncf
  first = (int)(((long long)2 * k * ncf - ncc + 2 * ncc - 1) / (2 * ncc));  // ceil((2k ncf - ncc) / 2ncc)
  if (first < 0) first = 0;
  last = (int)(((long long)2 * (k + 1) * ncf - ncc + 2 * ncc - 1) / (2 * ncc));
  if (last > ncf) last = ncf;
}

// Coarse cell modulus = mean of the fine cells whose centres it contains (nested: its 8
// children).
__global__ void cell_mean_kernel(const float* __restrict__ ef, int fcx, int fcy, int fcz,
                                 float* __restrict__ ec, int ccx, int ccy, int ccz) {
  const int64_t Nc = (int64_t)ccx * ccy * ccz;
  GRID_STRIDE(q, Nc) {
    const int I = (int)(q % ccx), J = (int)((q / ccx) % ccy), K = (int)(q / ((int64_t)ccx * ccy));
    int x0, x1, y0, y1, z0, z1;
    fine_cells_of(I, fcx, ccx, x0, x1);
    fine_cells_of(J, fcy, ccy, y0, y1);
    fine_cells_of(K, fcz, ccz, z0, z1);
    float s = 0.f;
    int cnt = 0;
    for (int kk = z0; kk < z1; kk++)
      for (int jj = y0; jj < y1; jj++)
        for (int ii = x0; ii < x1; ii++) {
          s += ef[((int64_t)kk * fcy + jj) * fcx + ii];
          cnt++;
        }
    ec[q] = cnt ? s / (float)cnt : 0.f;
  }
}

// r = dinv * (b - t), or dinv * b when t is null (x = 0); d = r / theta.
template <typename T>
__global__ void cheb_init_kernel(const T* __restrict__ b, const T* __restrict__ t,
                                 const T* __restrict__ dinv, T* __restrict__ r, T* __restrict__ d,
                                 const double* __restrict__ coef, int64_t n) {
  const T inv_theta = T(coef[1]);
  GRID_STRIDE(i, n) {
    const T ri = dinv[i] * (t ? b[i] - t[i] : b[i]);
    r[i] = ri;
    d[i] = ri * inv_theta;
  }
}

// x += d; and unless last: r -= dinv * t (t = K d); d = c1 d + c2 r, (c1, c2) = cf[0..1].
template <typename T>
__global__ void cheb_step_kernel(T* __restrict__ x, T* __restrict__ d, T* __restrict__ r,
                                 const T* __restrict__ t, const T* __restrict__ dinv,
                                 const double* __restrict__ cf, int last, int64_t n) {
  const T c1 = last ? T(0) : T(cf[0]), c2 = last ? T(0) : T(cf[1]);
  GRID_STRIDE(i, n) {
    const T di = d[i];
    x[i] += di;
    if (!last) {
      const T ri = r[i] - dinv[i] * t[i];
      r[i] = ri;
      d[i] = c1 * di + c2 * ri;
    }
  }
}

// Degree 1 (a Jacobi step weighted 1/theta) in one pass: x += dinv (b - t) / theta, or
// x = dinv b / theta from x = 0 (t null) -- cheb_init_kernel and the last
// cheb_step_kernel's arithmetic (the product rounded before the add, as there) without
// the r and d vectors.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <typename T>
__global__ void jacobi1_kernel(const T* __restrict__ b, const T* __restrict__ t,
                               const T* __restrict__ dinv, T* __restrict__ x,
                               const double* __restrict__ coef, int64_t n) {
  const T inv_theta = T(coef[1]);
  GRID_STRIDE(i, n) {
    const T di = mul_rn(dinv[i] * (t ? b[i] - t[i] : b[i]), inv_theta);
    x[i] = t ? x[i] + di : di;
  }
}

// The coarsest level's Chebyshev solve from x = 0 in one CTA (the level has <= 8 nodes
// per axis): the same iteration as chebyshev() with zero_start, its operator applied as
// one element per thread into shared memory (ncell x 8 x 3 values) and gathered per node
// in a fixed order, so the result is deterministic.  Replaces 2 deg launches.
constexpr int kCoarseThreads = 256, kCoarseMaxNodes = 8 * 8 * 8;
template <typename Op>
__global__ void __launch_bounds__(kCoarseThreads, 1)
    coarse_cheb_kernel(const typename Op::Args A0, const LayerTable L,
                       const typename Op::T* __restrict__ b, typename Op::T* __restrict__ x,
                       typename Op::T* __restrict__ r, typename Op::T* __restrict__ d,
                       const typename Op::T* __restrict__ dinv, const double* __restrict__ coef,
                       int deg) {
  using T = typename Op::T;
  extern __shared__ __align__(16) unsigned char coarse_smem[];
  T* yc = reinterpret_cast<T*>(coarse_smem);  // [cell][corner][component]
  typename Op::Args A = A0;
  A.x = d;
  const int nx = A.nx, ny = A.ny, nz = A.nz, cx = nx - 1, cy = ny - 1, cz = nz - 1;
  const int N = nx * ny * nz, ncell = cx * cy * cz;
  const T inv_theta = T(coef[1]);
  for (int n = threadIdx.x; n < N; n += blockDim.x)
    for (int c = 0; c < 3; c++) {
      const int i = 3 * n + c;
      const T ri = dinv[i] * b[i];
      r[i] = ri;
      d[i] = ri * inv_theta;
      x[i] = T(0);
    }
  for (int k = 0; k < deg; k++) {
    const bool last = k == deg - 1;
    if (!last) {
      __syncthreads();  // d complete
      for (int e = threadIdx.x; e < ncell; e += blockDim.x) {
        const int ex = e % cx, ey = (e / cx) % cy, ez = e / (cx * cy);
        T in[8][Op::NIN], out[8][Op::NC];
#pragma unroll
        for (int a = 0; a < 8; a++) {
          const typename Op::T* src[Op::NIN];
          Op::node_src(A, node_index(ex + (a & 1), ey + ((a >> 1) & 1), ez + (a >> 2), nx, ny), src);
#pragma unroll
          for (int q = 0; q < Op::NIN; q++) in[a][q] = *src[q];
        }
        Op::element(A, L, ex, ey, ez, in, out);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
          for (int c = 0; c < 3; c++) yc[(e * 8 + a) * 3 + c] = out[a][c];
      }
      __syncthreads();  // element values complete
    }
    const T c1 = last ? T(0) : T(coef[2 + 2 * k]), c2 = last ? T(0) : T(coef[3 + 2 * k]);
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
      const int i0 = n % nx, j0 = (n / nx) % ny, k0 = n / (nx * ny);
      T val[3] = {T(0), T(0), T(0)};
      if (!last)
        for (int dk = 0; dk < 2; dk++)
          for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) {
              const int ci = i0 - 1 + di, cj = j0 - 1 + dj, ck = k0 - 1 + dk;
              if (ci < 0 || cj < 0 || ck < 0 || ci >= cx || cj >= cy || ck >= cz) continue;
              const int a = (1 - di) + 2 * (1 - dj) + 4 * (1 - dk);
              const int e = (ck * cy + cj) * cx + ci;
              for (int c = 0; c < 3; c++) val[c] += yc[(e * 8 + a) * 3 + c];
            }
      const unsigned bb = A.bc ? A.bc[n] : 0u;
      for (int c = 0; c < 3; c++) {
        const int i = 3 * n + c;
        const T di = d[i];
        x[i] += di;
        if (!last) {
          const T t = ((bb >> c) & 1u) ? di : val[c];  // Dirichlet rows: t = d
          const T ri = r[i] - dinv[i] * t;
          r[i] = ri;
          d[i] = c1 * di + c2 * ri;
        }
      }
    }
  }
}

template <typename Op> size_t coarse_smem_bytes(int ncell) {
  return (size_t)ncell * 8 * 3 * sizeof(typename Op::T);
}

// The PCG step x += alpha p, r -= alpha w with alpha = rz / (p.w) formed on the device
// (pw = the dot product just reduced into *pw_in); nothing changes unless p.w > 0 (the
// host then stops on the indefinite or NaN p.w it reads back from pw_out).
__global__ void pcg_step_kernel(double* __restrict__ x, double* __restrict__ r,
                                const double* __restrict__ p, const double* __restrict__ w,
                                const double* __restrict__ pw_in, double* __restrict__ pw_out,
                                double rz, int64_t n) {
  const double pw = *pw_in;
  if (blockIdx.x == 0 && threadIdx.x == 0) *pw_out = pw;
  if (!(pw > 0.)) return;
  const double alpha = rz / pw;
  GRID_STRIDE(i, n) {
    x[i] += alpha * p[i];
    r[i] += (-alpha) * w[i];
  }
}

// Deterministic start vector of the power iteration in (-1/2, 1/2), 0 on Dirichlet dofs.
template <typename T>
__global__ void seed_kernel(T* __restrict__ x, const uint8_t* __restrict__ bc, int64_t N) {
  GRID_STRIDE(q, N) {
    const unsigned b = bc[q];
    for (int c = 0; c < 3; c++) {
      const uint64_t h = (uint64_t)(3 * q + c) * 0x9E3779B97F4A7C15ull;
      x[3 * q + c] = ((b >> c) & 1u) ? T(0) : T((double)((h >> 11) & 0xFFFFF) / 1048576.0 - 0.5);
    }
  }
}

// y = dinv * t; block partials of y.y and x.x (FP64) in partial[b], partial[nb + b].
template <typename T>
__global__ void __launch_bounds__(kPowThreads)
    power_dots_kernel(const T* __restrict__ t, const T* __restrict__ dinv, T* __restrict__ y,
                      const T* __restrict__ x, int64_t n, double* __restrict__ partial) {
  __shared__ double scratch[32];
  double yy = 0., xx = 0.;
  GRID_STRIDE(i, n) {
    const T yi = dinv[i] * t[i];
    y[i] = yi;
    yy += (double)yi * (double)yi;
    xx += (double)x[i] * (double)x[i];
  }
  const double syy = block_sum_dbl(yy, scratch);
  __syncthreads();
  const double sxx = block_sum_dbl(xx, scratch);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = syy;
    partial[gridDim.x + blockIdx.x] = sxx;
  }
}

// slot[0] = sqrt(y.y / x.x) (the eigenvalue estimate), slot[1] = 1 / |y| (0 if y = 0).
__global__ void __launch_bounds__(kPowThreads) power_final_kernel(const double* __restrict__ partial,
                                                                  int nb, double* __restrict__ slot) {
  __shared__ double scratch[32];
  double yy = 0., xx = 0.;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    yy += partial[b];
    xx += partial[nb + b];
  }
  const double syy = block_sum_dbl(yy, scratch);
  __syncthreads();
  const double sxx = block_sum_dbl(xx, scratch);
  if (threadIdx.x == 0) {
    slot[0] = sxx > 0. ? sqrt(syy / sxx) : 0.;
    slot[1] = syy > 0. ? 1. / sqrt(syy) : 0.;
  }
}

// x = y * slot[1]
template <typename T>
__global__ void power_norm_kernel(const T* __restrict__ y, T* __restrict__ x,
                                  const double* __restrict__ slot, int64_t n) {
  const T s = T(slot[1]);
  GRID_STRIDE(i, n) x[i] = y[i] * s;
}

// Chebyshev coefficients on [lo lmax, lmax], lmax = safety x estimate (Saad,
// Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 12.1):
// theta = (lmax + lmin) / 2, delta = (lmax - lmin) / 2, sigma = theta / delta,
// rho_0 = 1 / sigma, rho_{k+1} = 1 / (2 sigma - rho_k), c1 = rho_{k+1} rho_k,
// c2 = 2 rho_{k+1} / delta.  An estimate that is not positive leaves lmax = 0.
__global__ void cheb_coef_kernel(double* __restrict__ coef, int deg, double lo, double safety) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double est = coef[kCoefPerLevel - 2];
  const double lmax = est > 0. ? safety * est : 0.;
  coef[0] = lmax;
  const double lmin = lo * lmax, theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  if (!(lmax > 0.)) {
    for (int k = 1; k < kCoefPerLevel - 2; k++) coef[k] = 0.;
    return;
  }
  const double sigma = theta / delta;
  double rho = 1. / sigma;
  coef[1] = 1. / theta;
  for (int k = 0; k + 1 < deg; k++) {
    const double rho_new = 1. / (2. * sigma - rho);
    coef[2 + 2 * k] = rho_new * rho;
    coef[3 + 2 * k] = 2. * rho_new / delta;
    rho = rho_new;
  }
}

// ---------------------------------------------------------------------------------
// A level seen as a U operator in precision T.
template <typename T> void* dalloc(int64_t n, cudaError_t& e) {
  void* p = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&p, std::max<int64_t>(1, n) * sizeof(T));
  return p;
}

// Tabulates the transfer into level L from its finer neighbour (f nodes per axis):
// per axis pI, pw (f entries) and rlo, rn (L's node count entries), in L.xi / L.xw.
cudaError_t build_xfer(vfgpu_ctx::MGLevel& L, const int (&f)[3]) {
  const int c[3] = {L.nx, L.ny, L.nz};
  std::vector<int> xi;
  std::vector<double> xw;
  for (int d = 0; d < 3; d++) {  // pI, pw
    for (int i = 0; i < f[d]; i++) {
      const Lin l = fine_in_coarse(i, f[d], c[d]);
      xi.push_back(l.I);
      xw.push_back(l.whi);
    }
  }
  std::vector<int> rn;
  for (int d = 0; d < 3; d++) {  // rlo, rn: the fine nodes with a nonzero weight, an interval
    std::vector<int> lo(c[d], f[d]), hi(c[d], -1);
    for (int i = 0; i < f[d]; i++) {
      const Lin l = fine_in_coarse(i, f[d], c[d]);
      lo[l.I] = std::min(lo[l.I], i);
      hi[l.I] = std::max(hi[l.I], i);
      if (l.whi > 0.0) {
        lo[l.I + 1] = std::min(lo[l.I + 1], i);
        hi[l.I + 1] = std::max(hi[l.I + 1], i);
      }
    }
    for (int I = 0; I < c[d]; I++) {
      if (hi[I] < lo[I] || hi[I] - lo[I] >= 4) return cudaErrorInvalidValue;
      xi.push_back(lo[I]);
      rn.push_back(hi[I] - lo[I] + 1);
    }
  }
  xi.insert(xi.end(), rn.begin(), rn.end());  // the order xfer_of reads
  if (xi.size() != (size_t)(f[0] + f[1] + f[2]) + 2 * (size_t)(c[0] + c[1] + c[2]))
    return cudaErrorInvalidValue;
  cudaError_t e = cudaSuccess;
  L.xi = (int*)dalloc<int>((int64_t)xi.size(), e);
  L.xw = (double*)dalloc<double>((int64_t)xw.size(), e);
  if (e == cudaSuccess) e = cudaMemcpy(L.xi, xi.data(), xi.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(L.xw, xw.data(), xw.size() * sizeof(double), cudaMemcpyHostToDevice);
  return e;
}

// The transfer tables of level l (from level l - 1) as kernel arguments.
Xfer xfer_of(vfgpu_ctx* c, int l) {
  const auto& L = c->mg[l];
  const auto& F = c->mg[l - 1];
  const int f[3] = {F.nx, F.ny, F.nz}, n[3] = {L.nx, L.ny, L.nz};
  Xfer X;
  int oi = 0, ow = 0;
  for (int d = 0; d < 3; d++) {
    X.a[d].pI = L.xi + oi;
    X.a[d].pw = L.xw + ow;
    oi += f[d];
    ow += f[d];
  }
  for (int d = 0; d < 3; d++) {
    X.a[d].rlo = L.xi + oi;
    oi += n[d];
  }
  for (int d = 0; d < 3; d++) {
    X.a[d].rn = L.xi + oi;
    oi += n[d];
  }
  for (int d = 0; d < 3; d++) {
    X.a[d].nf = f[d];
    X.a[d].mode = n[d] == f[d] ? kXferIdentity : (f[d] - 1 == 2 * (n[d] - 1) ? kXferNested : kXferTable);
  }
  return X;
}

template <typename T> struct LevelT {
  int nx, ny, nz;
  double hx, hy, hz;
  const TilePlan* plan;
  T* seam;
  const T* v;
  const uint8_t* bc;
  const uint8_t* elayer;
  const float* cellE;
  const T* dinv;
  const uint32_t* cflag;  // fine level under NOCOMPRESSION: the Jacobian's bits
  vfgpu::UnitLists ul;    // fine level: the ctx's unit lists of its plan (else none)
  T *x, *b, *r, *d, *t;
  double* coef;
  int64_t n3;
};

template <typename T> const TilePlan* fine_plan(vfgpu_ctx* c);
template <> const TilePlan* fine_plan<double>(vfgpu_ctx* c) { return &c->plan64; }
template <> const TilePlan* fine_plan<float>(vfgpu_ctx* c) { return &c->plan32; }
template <typename T> T* fine_seam(vfgpu_ctx* c);
template <> double* fine_seam<double>(vfgpu_ctx* c) { return c->seam64; }
template <> float* fine_seam<float>(vfgpu_ctx* c) { return c->seam32; }
template <typename T> const T* fine_v(vfgpu_ctx* c);
template <> const double* fine_v<double>(vfgpu_ctx* c) { return c->f[VFGPU_FIELD_V]; }
template <> const float* fine_v<float>(vfgpu_ctx* c) { return c->V32; }

template <typename T> LevelT<T> view(vfgpu_ctx* c, int l) {
  auto& L = c->mg[l];
  LevelT<T> V;
  V.x = (T*)L.x;
  V.b = (T*)L.b;
  V.r = (T*)L.r;
  V.d = (T*)L.d;
  V.t = (T*)L.t;
  V.coef = L.coef;
  if (l == 0) {
    V.nx = c->nx;
    V.ny = c->ny;
    V.nz = c->nz;
    V.hx = c->hx;
    V.hy = c->hy;
    V.hz = c->hz;
    V.plan = fine_plan<T>(c);
    V.seam = fine_seam<T>(c);
    V.v = fine_v<T>(c);
    V.bc = c->bcU_bits;
    V.elayer = c->d_elayer;
    V.cellE = c->d_cellE;
    V.dinv = (const T*)c->mg_dinv0;
    V.cflag = c->unilateral ? c->d_cflag : nullptr;
    V.ul = u_lists_on(c, (int)sizeof(T)) ? (sizeof(T) == 8 ? c->ul64 : c->ul32) : UnitLists{};
    V.n3 = 3 * c->N;
  } else {
    V.nx = L.nx;
    V.ny = L.ny;
    V.nz = L.nz;
    V.hx = L.hx;
    V.hy = L.hy;
    V.hz = L.hz;
    V.plan = &L.plan;
    V.seam = (T*)L.seam;
    V.v = (const T*)L.v;
    V.bc = L.bc;
    V.elayer = L.elayer;
    V.cellE = L.cellE;
    V.dinv = (const T*)L.dinv;
    V.cflag = nullptr;
    V.ul = UnitLists{};
    V.n3 = 3 * L.N;
  }
  return V;
}

template <typename T> UApplyArgs<T> level_args(vfgpu_ctx* c, const LevelT<T>& V, const T* x, T* y) {
  UApplyArgs<T> A{};
  A.x = x;
  A.v = V.v;
  A.y = y;
  A.bc = V.bc;
  A.elayer = V.elayer;
  A.cellE = V.cellE;
  A.seamX = V.seam;
  A.seamY = V.seam + V.plan->seamX;
  A.nx = V.nx;
  A.ny = V.ny;
  A.nz = V.nz;
  A.ihx = T(1.0 / V.hx);
  A.ihy = T(1.0 / V.hy);
  A.ihz = T(1.0 / V.hz);
  A.vol = T(V.hx * V.hy * V.hz);
  A.eta = T(c->vf.eta);
  A.P = c->d_params;
  A.cflag = V.cflag;
  use_unit_lists(A, V.ul);
  A.plane_err = c->d_cerr;
  return A;
}

template <typename T>
cudaError_t level_apply(vfgpu_ctx* c, const LevelT<T>& V, const T* x, T* y) {
  return launch_u_apply<T>(level_args<T>(c, V, x, y), *V.plan, c->layers, c->stream);
}

// Chebyshev iteration on D^-1 K x = D^-1 b with the level's coefficients; x updated in
// place (zero_start: x = 0 on entry and no initial residual apply).  (Carrying the
// update in the operator's epilogue instead of a separate pass measured slower on B200:
// StepU 257^3 0.250 s against 0.225 s mixed, 0.378 s against 0.328 s FP64 -- the extra
// loads stall the compute-bound z-march.)
template <typename T>
cudaError_t chebyshev(vfgpu_ctx* c, const LevelT<T>& V, const T* b, T* x, int deg, bool zero_start) {
  const int64_t n3 = V.n3;
  if (deg == 1) {
    cudaError_t e = zero_start ? cudaSuccess : level_apply<T>(c, V, x, V.t);
    if (e == cudaSuccess) {
      jacobi1_kernel<T><<<blocks_for(n3), 256, 0, c->stream>>>(b, zero_start ? nullptr : V.t, V.dinv,
                                                              x, V.coef, n3);
      e = cudaGetLastError();
    }
    return e;
  }
  cudaError_t e =
      zero_start ? cudaMemsetAsync(x, 0, n3 * sizeof(T), c->stream) : level_apply<T>(c, V, x, V.t);
  if (e == cudaSuccess) {
    cheb_init_kernel<T><<<blocks_for(n3), 256, 0, c->stream>>>(b, zero_start ? nullptr : V.t, V.dinv,
                                                              V.r, V.d, V.coef, n3);
    e = cudaGetLastError();
  }
  for (int k = 0; k < deg && e == cudaSuccess; k++) {
    const bool last = k == deg - 1;
    if (!last) e = level_apply<T>(c, V, V.d, V.t);
    if (e == cudaSuccess) {
      cheb_step_kernel<T><<<blocks_for(n3), 256, 0, c->stream>>>(x, V.d, V.r, V.t, V.dinv,
                                                                V.coef + 2 + 2 * k, last ? 1 : 0, n3);
      e = cudaGetLastError();
    }
  }
  return e;
}

// The coarsest level's solve: kCoarseDeg Chebyshev steps from x = 0, in one CTA.
template <typename T> cudaError_t coarse_solve(vfgpu_ctx* c, const LevelT<T>& V, const T* b, T* x) {
  if (V.n3 / 3 > kCoarseMaxNodes || V.cflag) return chebyshev<T>(c, V, b, x, kCoarseDeg, true);
  const UApplyArgs<T> A = level_args<T>(c, V, V.d, V.t);
  const int ncell = (V.nx - 1) * (V.ny - 1) * (V.nz - 1);
  if (A.ihx == A.ihy && A.ihy == A.ihz)
    coarse_cheb_kernel<UOp<T, true>>
        <<<1, kCoarseThreads, coarse_smem_bytes<UOp<T, true>>(ncell), c->stream>>>(
            A, c->layers, b, x, V.r, V.d, V.dinv, V.coef, kCoarseDeg);
  else
    coarse_cheb_kernel<UOp<T>><<<1, kCoarseThreads, coarse_smem_bytes<UOp<T>>(ncell), c->stream>>>(
        A, c->layers, b, x, V.r, V.d, V.dinv, V.coef, kCoarseDeg);
  return cudaGetLastError();
}

// Lets the coarsest solve take the shared memory of an 8 x 8 x 8 level.
template <typename T> cudaError_t coarse_attributes() {
  const int ncell = (8 - 1) * (8 - 1) * (8 - 1);
  cudaError_t e = cudaFuncSetAttribute(coarse_cheb_kernel<UOp<T, true>>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)coarse_smem_bytes<UOp<T, true>>(ncell));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(coarse_cheb_kernel<UOp<T>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)coarse_smem_bytes<UOp<T>>(ncell));
  return e;
}

// z = V-cycle(b) from level l down.
template <typename T> cudaError_t vcycle(vfgpu_ctx* c, int l, const T* b, T* z) {
  const LevelT<T> V = view<T>(c, l);
  if (l == (int)c->mg.size() - 1) return coarse_solve<T>(c, V, b, z);
  const LevelT<T> C = view<T>(c, l + 1);
  cudaError_t e = chebyshev<T>(c, V, b, z, kSmoothDeg, true);
  if (e == cudaSuccess) e = level_apply<T>(c, V, z, V.t);
  if (e == cudaSuccess) {
    restrict_kernel<T><<<blocks_for(C.n3 / 3), 256, 0, c->stream>>>(
        b, V.t, V.bc, V.nx, V.ny, xfer_of(c, l + 1), C.b, C.nx, C.ny, C.nz, C.bc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = vcycle<T>(c, l + 1, C.b, C.x);
  if (e == cudaSuccess) {
    prolong_add_kernel<T><<<blocks_for(V.n3 / 3), 256, 0, c->stream>>>(
        C.x, C.nx, C.ny, xfer_of(c, l + 1), z, V.nx, V.ny, V.nz, V.bc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = chebyshev<T>(c, V, b, z, kSmoothDeg, false);
  return e;
}

// Next coarser node count along an axis: ceil(cells / 2) cells while the axis keeps
// >= 5 nodes, else unchanged.
inline int coarser(int n) { return n >= 9 ? n / 2 + 1 : n; }
// Levels of the hierarchy of an nx x ny x nz grid (1: no coarse level).
inline int mg_levels(int nx, int ny, int nz) {
  int nlev = 1;
  while (coarser(nx) != nx || coarser(ny) != ny || coarser(nz) != nz) {
    nx = coarser(nx);
    ny = coarser(ny);
    nz = coarser(nz);
    nlev++;
  }
  return nlev;
}
// First fine cell (along one axis) whose centre lies in coarse cell k (host mirror of
// fine_cells_of).
inline int first_fine_cell(int k, int ncf, int ncc) {
  const long long a = 2LL * k * ncf - ncc, b = 2LL * ncc;
  return a <= 0 ? 0 : (int)((a + b - 1) / b);
}

// Allocates the hierarchy in precision T (rebuilt when the precision changes).
template <typename T> int mg_build(vfgpu_ctx* c) {
  if (!c->mg.empty() && c->mg_bytes == (int)sizeof(T)) return VFGPU_OK;
  free_mg(c);
  const int nlev = mg_levels(c->nx, c->ny, c->nz);
  if (nlev < 2) return fail(VFGPU_ERR_INVALID, "multigrid needs >= 9 nodes along some axis");
  cudaError_t e = coarse_attributes<T>();
  c->mg_coef = (double*)dalloc<double>((int64_t)kCoefPerLevel * nlev, e);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->mg_coef, 0, sizeof(double) * kCoefPerLevel * nlev, c->stream);
  const bool f32 = sizeof(T) == 4;
  c->mg.resize(nlev);
  {
    auto& L0 = c->mg[0];
    const int64_t n3 = 3 * c->N;
    L0.nx = c->nx;
    L0.ny = c->ny;
    L0.nz = c->nz;
    L0.N = c->N;
    L0.NC = c->NC;
    // FP32: r and d also hold the FP64 diagonal of each coarse level during set-up
    const int64_t n1 = (int64_t)coarser(c->nx) * coarser(c->ny) * coarser(c->nz);
    const int64_t nrd = f32 ? std::max<int64_t>(n3, 6 * n1) : n3;
    L0.x = dalloc<T>(n3, e);
    L0.ev = dalloc<T>(n3, e);
    L0.r = dalloc<T>(nrd, e);
    L0.d = dalloc<T>(nrd, e);
    L0.t = dalloc<T>(n3, e);
    if (f32) {
      L0.b = dalloc<T>(n3, e);
      c->mg_z = (double*)dalloc<double>(n3, e);
    }
    L0.coef = c->mg_coef;
  }
  int nx = c->nx, ny = c->ny, nz = c->nz;
  for (int l = 1; l < nlev && e == cudaSuccess; l++) {
    const int f[3] = {nx, ny, nz};
    nx = coarser(nx);
    ny = coarser(ny);
    nz = coarser(nz);
    const double hx = c->lx / (nx - 1), hy = c->ly / (ny - 1), hz = c->lz / (nz - 1);
    auto& L = c->mg[l];
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.N = (int64_t)nx * ny * nz;
    L.NC = (int64_t)(nx - 1) * (ny - 1) * (nz - 1);
    L.hx = hx;
    L.hy = hy;
    L.hz = hz;
    L.plan = u_plan(nx, ny, nz, (int)sizeof(T), c->nsm);
    L.seam = dalloc<T>((int64_t)(L.plan.seamX + L.plan.seamY), e);
    for (void** p : {&L.x, &L.b, &L.r, &L.d, &L.t, &L.dinv, &L.ev}) *p = dalloc<T>(3 * L.N, e);
    L.v64 = (double*)dalloc<double>(L.N, e);
    L.v = f32 ? dalloc<float>(L.N, e) : (void*)L.v64;
    L.bc = (uint8_t*)dalloc<uint8_t>(L.N, e);
    L.elayer = (uint8_t*)dalloc<uint8_t>(nz - 1, e);
    if (c->d_cellE) L.cellE = (float*)dalloc<float>(L.NC, e);
    etab_host(hx, hy, hz, &L.tab);
    L.coef = c->mg_coef + (int64_t)kCoefPerLevel * l;
    if (e == cudaSuccess) e = build_xfer(L, f);
  }
  c->mg_bytes = (int)sizeof(T);
  c->mg_ready = false;
  c->mg_layers = false;
  if (e != cudaSuccess) {
    free_mg(c);
    return cuda_fail(e, "multigrid hierarchy");
  }
  return VFGPU_OK;
}

// Per operator: coarse fields from the fine ones, diagonals, eigenvalue bounds and
// Chebyshev coefficients.
template <typename T> int mg_setup(vfgpu_ctx* c) {
  cudaError_t e = cudaSuccess;
  const bool f32 = sizeof(T) == 4;
  const int nlev = (int)c->mg.size();
  for (int l = 1; l < nlev && e == cudaSuccess; l++) {  // set_cell_modulus after the build
    auto& L = c->mg[l];
    if (c->d_cellE && !L.cellE) e = cudaMalloc((void**)&L.cellE, L.NC * sizeof(float));
  }
  // element layers of the coarse levels: the layer of the lowest fine layer in each
  // coarse layer, followed down to level 0 (uploaded once per hierarchy and material)
  if (!c->mg_layers) {
    std::vector<uint8_t> el(std::max(1, c->nz - 1));
    if (e == cudaSuccess) e = cudaMemcpyAsync(el.data(), c->d_elayer, el.size(), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    std::vector<std::vector<uint8_t>> all(nlev);
    for (int l = 1; l < nlev && e == cudaSuccess; l++) {
      auto& L = c->mg[l];
      all[l].resize(L.nz - 1);
      for (int k = 0; k < L.nz - 1; k++) {
        int kk = k;
        for (int m = l; m >= 1; m--) kk = first_fine_cell(kk, c->mg[m - 1].nz - 1, c->mg[m].nz - 1);
        all[l][k] = el[std::min<size_t>(kk, el.size() - 1)];
      }
      e = cudaMemcpyAsync(L.elayer, all[l].data(), all[l].size(), cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // the host copies leave scope
    if (e == cudaSuccess) c->mg_layers = true;
  }
  for (int l = 1; l < nlev && e == cudaSuccess; l++) {
    auto& L = c->mg[l];
    auto& F = c->mg[l - 1];
    const double* vf = l == 1 ? c->f[VFGPU_FIELD_V] : F.v64;
    const uint8_t* bcf = l == 1 ? c->bcU_bits : F.bc;
    const float* cellEf = l == 1 ? c->d_cellE : F.cellE;
    const int fx = l == 1 ? c->nx : F.nx, fy = l == 1 ? c->ny : F.ny, fz = l == 1 ? c->nz : F.nz;
    inject_kernel<<<blocks_for(L.N), 256, 0, c->stream>>>(vf, bcf, fx, fy, fz, L.v64, L.bc, L.nx,
                                                          L.ny, L.nz);
    e = cudaGetLastError();
    if (e == cudaSuccess && f32) e = convert_f64_f32(L.v64, (float*)L.v, L.N, c->stream);
    if (e == cudaSuccess && c->d_cellE) {
      cell_mean_kernel<<<blocks_for(L.NC), 256, 0, c->stream>>>(cellEf, fx - 1, fy - 1, fz - 1,
                                                               L.cellE, L.nx - 1, L.ny - 1,
                                                               L.nz - 1);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      // FP64 diagonal; FP32 hierarchy: computed in the fine level's FP32 work vectors r
      // and d, allocated with >= 24 N_1 bytes each
      double* diag = f32 ? (double*)c->mg[0].r : (double*)L.t;
      double* dinv64 = f32 ? (double*)c->mg[0].d : (double*)L.dinv;
      ElemArgs E{};
      E.tab = L.tab;
      E.nx = L.nx;
      E.ny = L.ny;
      E.nz = L.nz;
      E.elayer = L.elayer;
      E.cellE = c->d_cellE ? L.cellE : nullptr;
      E.L = c->layers;
      E.eta = c->vf.eta;
      E.hx = L.hx;
      E.hy = L.hy;
      E.hz = L.hz;
      e = launch_u_diag(E, L.v64, L.bc, diag, c->stream);
      if (e == cudaSuccess) e = dev_inv(diag, dinv64, f32 ? (float*)L.dinv : nullptr, 3 * L.N, c->stream);
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "multigrid set-up");
  // largest eigenvalue of D^-1 K per level by power iteration, then the coefficients
  for (int l = 0; l < nlev && e == cudaSuccess; l++) {
    const LevelT<T> V = view<T>(c, l);
    double* slot = V.coef + kCoefPerLevel - 2;
    T* ev = (T*)c->mg[l].ev;
    if (!c->mg_ev) {
      seed_kernel<T><<<blocks_for(V.n3 / 3), 256, 0, c->stream>>>(ev, V.bc, V.n3 / 3);
      e = cudaGetLastError();
    }
    const int its = c->mg_ev ? kWarmPowerIts : kPowerIts;
    for (int it = 0; it < its && e == cudaSuccess; it++) {
      e = level_apply<T>(c, V, ev, V.t);
      if (e == cudaSuccess) {
        power_dots_kernel<T><<<kPowBlocks, kPowThreads, 0, c->stream>>>(V.t, V.dinv, V.d, ev, V.n3,
                                                                       c->d_red);
        power_final_kernel<<<1, kPowThreads, 0, c->stream>>>(c->d_red, kPowBlocks, slot);
        power_norm_kernel<T><<<blocks_for(V.n3), 256, 0, c->stream>>>(V.d, ev, slot, V.n3);
        e = cudaGetLastError();
      }
    }
    if (e == cudaSuccess) {
      const bool last = l == nlev - 1;
      cheb_coef_kernel<<<1, 32, 0, c->stream>>>(V.coef, last ? kCoarseDeg : kSmoothDeg,
                                                last ? kCoarseLo : kSmoothLo, kLmaxSafety);
      e = cudaGetLastError();
    }
  }
  std::vector<double> coef((size_t)kCoefPerLevel * nlev);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(coef.data(), c->mg_coef, coef.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "multigrid eigenvalue estimate");
  for (int l = 0; l < nlev; l++)
    if (!(coef[(size_t)kCoefPerLevel * l] > 0.) || !std::isfinite(coef[(size_t)kCoefPerLevel * l])) {
      c->mg_ev = false;  // reseed next time
      return fail(VFGPU_ERR_STATE, "multigrid: no positive eigenvalue estimate on level %d", l);
    }
  c->mg_ready = true;
  c->mg_ev = true;
  return VFGPU_OK;
}

// One preconditioner application z = M^-1 r (FP64 in and out), as a graph replay.
template <typename T> cudaError_t precondition(vfgpu_ctx* c, const double* r, double* z);
template <> cudaError_t precondition<double>(vfgpu_ctx* c, const double* r, double* z) {
  auto body = [c, r, z]() { return vcycle<double>(c, 0, r, z); };
  cudaGraphExec_t g = c->use_graphs ? ctx_graph(c, kGraphMG64, 0, body) : nullptr;
  return g ? cudaGraphLaunch(g, c->stream) : body();
}
template <> cudaError_t precondition<float>(vfgpu_ctx* c, const double* r, double* z) {
  auto body = [c, r, z]() {
    const LevelT<float> V = view<float>(c, 0);
    cudaError_t e = convert_f64_f32(r, V.b, V.n3, c->stream);
    if (e == cudaSuccess) e = vcycle<float>(c, 0, V.b, V.x);
    if (e == cudaSuccess) e = convert_f32_f64(V.x, z, V.n3, c->stream);
    return e;
  };
  cudaGraphExec_t g = c->use_graphs ? ctx_graph(c, kGraphMG32, 0, body) : nullptr;
  return g ? cudaGraphLaunch(g, c->stream) : body();
}

template <typename T>
int mgcg(vfgpu_ctx* c, const double* b, double* x, double* r, double* p, double* w,
         const double* dinv0, bool reuse, double rtol, double atol, double dtol, int maxit,
         int* its, int* reason, int* levels) {
  int rc = mg_build<T>(c);
  if (rc) return rc;
  if (!reuse || !c->mg_ready) {
    rc = mg_setup<T>(c);
    if (rc) return rc;
  }
  *levels = (int)c->mg.size();
  const int64_t n3 = 3 * c->N;
  // the preconditioned residual: the V-cycle's own output vector in FP64
  double* z = sizeof(T) == 8 ? (double*)c->mg[0].x : c->mg_z;
  cudaError_t e = cudaMemsetAsync(x, 0, n3 * sizeof(double), c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(r, b, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  // h[0] = r.z, h[2] = ||D^-1 r||^2, h[8] = the step's p.w (one host read per iteration)
  double h[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
  auto scalars = [&]() {
    const double* pa[1] = {r};
    const double* pb[1] = {z};
    if (e == cudaSuccess) e = dev_dots(pa, pb, 1, n3, c->d_red, c->d_out, c->stream);
    if (e == cudaSuccess) e = dev_znorm2(r, dinv0, n3, c->d_red, c->d_out + 2, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, c->d_out, 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  };
  if (e == cudaSuccess) e = precondition<T>(c, r, z);
  scalars();
  if (e != cudaSuccess) return cuda_fail(e, "multigrid PCG");
  double rz = h[0];
  const double rnorm0 = sqrt(h[2]), ttol = std::max(rtol * rnorm0, atol);
  *its = 0;
  *reason = 0;
  if (!(rnorm0 == rnorm0)) *reason = CG_DIVERGED_NAN;
  else if (rnorm0 <= ttol) *reason = rnorm0 <= atol ? CG_CONVERGED_ATOL : CG_CONVERGED_RTOL;
  else if (!(rz > 0.)) *reason = rz == 0. ? CG_CONVERGED_ATOL : CG_DIVERGED_INDEFINITE;
  if (!*reason) e = cudaMemcpyAsync(p, z, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  LevelT<double> outer{};  // the FP64 Jacobian whatever the V-cycle's precision
  outer.nx = c->nx;
  outer.ny = c->ny;
  outer.nz = c->nz;
  outer.hx = c->hx;
  outer.hy = c->hy;
  outer.hz = c->hz;
  outer.plan = &c->plan64;
  outer.seam = c->seam64;
  outer.v = c->f[VFGPU_FIELD_V];
  outer.bc = c->bcU_bits;
  outer.elayer = c->d_elayer;
  outer.cellE = c->d_cellE;
  outer.cflag = c->unilateral ? c->d_cflag : nullptr;
  outer.ul = u_lists_on(c, 8) ? c->ul64 : UnitLists{};
  while (!*reason && e == cudaSuccess) {
    e = level_apply<double>(c, outer, p, w);
    const double* pa[1] = {p};
    const double* pb[1] = {w};
    if (e == cudaSuccess) e = dev_dots(pa, pb, 1, n3, c->d_red, c->d_out, c->stream);
    if (e == cudaSuccess) {
      pcg_step_kernel<<<blocks_for(n3), 256, 0, c->stream>>>(x, r, p, w, c->d_out, c->d_out + 8, rz, n3);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = precondition<T>(c, r, z);
    scalars();
    if (e != cudaSuccess) break;
    const double pw = h[8];
    if (!(pw > 0.)) {  // x and r were left unchanged
      *reason = (pw == pw) ? CG_DIVERGED_INDEFINITE : CG_DIVERGED_NAN;
      break;
    }
    *its += 1;
    const double dp = sqrt(h[2]);
    if (!(dp == dp)) *reason = CG_DIVERGED_NAN;
    else if (dp <= ttol) *reason = CG_CONVERGED_RTOL;
    else if (dp >= dtol * rnorm0) *reason = CG_DIVERGED_DTOL;
    else if (*its >= maxit) *reason = CG_DIVERGED_ITS;
    else if (!(h[0] > 0.)) *reason = h[0] == 0. ? CG_CONVERGED_ATOL : CG_DIVERGED_INDEFINITE;
    else {
      const double beta = h[0] / rz;
      rz = h[0];
      e = dev_axpby(p, z, beta, p, n3, c->stream);  // p = z + beta p
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "multigrid PCG");
  return VFGPU_OK;
}

}  // namespace

void free_mg(vfgpu_ctx* c) {
  for (size_t k = 0; k < c->graphs.size();) {  // the V-cycle graphs hold the old pointers
    auto& g = c->graphs[k];
    if (g.kind == kGraphMG64 || g.kind == kGraphMG32) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      c->graphs.erase(c->graphs.begin() + k);
    } else {
      k++;
    }
  }
  for (auto& L : c->mg) {
    void* bufs[] = {L.seam, L.x, L.b, L.r, L.d, L.t, L.dinv, L.ev, L.bc, L.elayer, L.cellE,
                    L.xi, L.xw};
    for (void* p : bufs) cudaFree(p);
    if (L.v != (void*)L.v64) cudaFree(L.v);
    cudaFree(L.v64);
  }
  c->mg.clear();
  cudaFree(c->mg_coef);
  cudaFree(c->mg_z);
  c->mg_coef = nullptr;
  c->mg_z = nullptr;
  c->mg_bytes = 0;
  c->mg_ready = false;
  c->mg_ev = false;
}

long long mg_memory_bytes(int nx, int ny, int nz, int bytes) {
  const long long N = (long long)nx * ny * nz;
  const long long N1 = (long long)coarser(nx) * coarser(ny) * coarser(nz);
  const long long nrd = bytes == 4 ? std::max(3 * N, 6 * N1) : 3 * N;
  long long b = (3 * 3 * N + 2 * nrd) * bytes + (bytes == 4 ? 3 * N * (4 + 8) : 0);  // fine vectors
  const int nlev = mg_levels(nx, ny, nz);
  for (int l = 1; l < nlev; l++) {
    b += (long long)(nx + ny + nz) * (4 + 8);  // transfer tables
    nx = coarser(nx);
    ny = coarser(ny);
    nz = coarser(nz);
    b += (long long)(nx + ny + nz) * 8;
    const long long Nl = (long long)nx * ny * nz, NCl = (long long)(nx - 1) * (ny - 1) * (nz - 1);
    const TilePlan p = u_plan(nx, ny, nz, bytes, 148);
    b += (long long)(p.seamX + p.seamY) * bytes + 7 * 3 * Nl * bytes + Nl * 8 +
         (bytes == 4 ? Nl * 4 : 0) + Nl + (nz - 1) + NCl * 4;
  }
  if (nlev < 2) return 0;
  return b + (long long)kCoefPerLevel * nlev * 8;
}

int run_mgcg(vfgpu_ctx* c, bool fp32, const double* b, double* x, double* r, double* p, double* w,
             const double* dinv0, const float* dinv0_32, bool reuse, double rtol, double atol,
             double dtol, int maxit, int* its, int* reason, int* levels) {
  c->mg_dinv0 = fp32 ? (const void*)dinv0_32 : (const void*)dinv0;
  if (fp32)
    return mgcg<float>(c, b, x, r, p, w, dinv0, reuse, rtol, atol, dtol, maxit, its, reason, levels);
  return mgcg<double>(c, b, x, r, p, w, dinv0, reuse, rtol, atol, dtol, maxit, its, reason, levels);
}

}  // namespace vfgpu

extern "C" int vfgpu_mg_hierarchy(const vfgpu_grid* g, int bytes, int max_levels, int* dims,
                                  int* nlevels, long long* mg_bytes) {
  if (!g || !nlevels || (max_levels > 0 && !dims) || (bytes != 4 && bytes != 8))
    return vfgpu::fail(VFGPU_ERR_INVALID, "vfgpu_mg_hierarchy: bad argument");
  if (g->nx < 2 || g->ny < 2 || g->nz < 2)
    return vfgpu::fail(VFGPU_ERR_INVALID, "vfgpu_mg_hierarchy: bad grid");
  int nx = g->nx, ny = g->ny, nz = g->nz;
  const int nlev = vfgpu::mg_levels(nx, ny, nz);
  for (int l = 0; l < nlev && l < max_levels; l++) {
    dims[3 * l] = nx;
    dims[3 * l + 1] = ny;
    dims[3 * l + 2] = nz;
    nx = vfgpu::coarser(nx);
    ny = vfgpu::coarser(ny);
    nz = vfgpu::coarser(nz);
  }
  *nlevels = nlev;
  if (mg_bytes) *mg_bytes = vfgpu::mg_memory_bytes(g->nx, g->ny, g->nz, bytes);
  return VFGPU_OK;
}
