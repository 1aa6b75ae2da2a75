// mg.cu -- geometric multigrid V-cycle as the preconditioner of the U solve's CG
// (solve option VFGPU_PC_MG).  No counterpart in the reference, whose snesU uses
// KSPCG with Jacobi (or hypre when PETSc has it, VFCommon.c:1044-1047); the solve it
// feeds keeps the reference's semantics (same residual, same SNES tests), only the
// Krylov iterations get fewer.
//
// Levels halve the cells per axis while every axis has an even cell count and the
// coarse grid keeps >= 5 nodes per axis.  Each coarse level rediscretises the same
// operator (the tile engine's U apply) on its grid with the phase field injected
// from the level above (v_c(I) = v_f(2I)), the Dirichlet bits injected the same
// way, the element layer of the lower child layer and, for a per-cell modulus, the
// mean of the 8 children.  Transfers: trilinear prolongation and its transpose
// (full weighting), Dirichlet dofs zeroed after each.  Smoother: Chebyshev
// iteration of D^-1 K of degree 3 on [lmax/10, lmax] (lmax from 12 power
// iterations per level and solve), pre and post; the coarsest level runs degree 30
// on [lmax/100, lmax].  Everything is a fixed sequence of deterministic kernels, so
// the V-cycle is a fixed symmetric linear operator and plain PCG applies.
#include <algorithm>
#include <cmath>
#include <vector>

#include "abi_util.h"
#include "solver.h"
#include "vec.h"

namespace vfgpu {
namespace {

constexpr int kSmoothDeg = 3, kCoarseDeg = 30, kPowerIts = 12;
constexpr double kSmoothLo = 0.1, kCoarseLo = 0.01;

inline int blocks_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

#define GRID_STRIDE(i, n)                                                                \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n);              \
       i += (int64_t)gridDim.x * blockDim.x)

// Full weighting: coarse node I gathers the fine nodes 2I + o, o in {-1,0,1}^3, with
// weight prod_d (1 - |o_d| / 2), skipping fine Dirichlet dofs; Dirichlet dofs of the
// coarse level are zeroed.  This is the transpose of prolong_add_kernel.
__global__ void restrict_kernel(const double* __restrict__ rf, const uint8_t* __restrict__ bc_f,
                                int fx, int fy, int fz, double* __restrict__ rc, int cx, int cy,
                                int cz, const uint8_t* __restrict__ bc_c) {
  const int64_t Nc = (int64_t)cx * cy * cz;
  GRID_STRIDE(q, Nc) {
    const int I = (int)(q % cx), J = (int)((q / cx) % cy), K = (int)(q / ((int64_t)cx * cy));
    double acc[3] = {0., 0., 0.};
    for (int oz = -1; oz <= 1; oz++) {
      const int k = 2 * K + oz;
      if (k < 0 || k >= fz) continue;
      const double wz = oz ? 0.5 : 1.0;
      for (int oy = -1; oy <= 1; oy++) {
        const int j = 2 * J + oy;
        if (j < 0 || j >= fy) continue;
        const double wy = oy ? 0.5 : 1.0;
        for (int ox = -1; ox <= 1; ox++) {
          const int i = 2 * I + ox;
          if (i < 0 || i >= fx) continue;
          const double w = wz * wy * (ox ? 0.5 : 1.0);
          const int64_t n = node_index(i, j, k, fx, fy);
          const unsigned bf = bc_f[n];
          for (int c = 0; c < 3; c++)
            if (!((bf >> c) & 1u)) acc[c] += w * rf[3 * n + c];
        }
      }
    }
    const unsigned b = bc_c[q];
    for (int c = 0; c < 3; c++) rc[3 * q + c] = ((b >> c) & 1u) ? 0. : acc[c];
  }
}

// x_f += trilinear interpolation of e_c (fine Dirichlet dofs untouched: they stay 0).
__global__ void prolong_add_kernel(const double* __restrict__ ec, int cx, int cy,
                                   double* __restrict__ xf, int fx, int fy, int fz,
                                   const uint8_t* __restrict__ bc_f) {
  const int64_t Nf = (int64_t)fx * fy * fz;
  GRID_STRIDE(q, Nf) {
    const int i = (int)(q % fx), j = (int)((q / fx) % fy), k = (int)(q / ((int64_t)fx * fy));
    const int i0 = i >> 1, j0 = j >> 1, k0 = k >> 1;
    const int ni = (i & 1) ? 2 : 1, nj = (j & 1) ? 2 : 1, nk = (k & 1) ? 2 : 1;
    const double wi = (i & 1) ? 0.5 : 1.0, wj = (j & 1) ? 0.5 : 1.0, wk = (k & 1) ? 0.5 : 1.0;
    double acc[3] = {0., 0., 0.};
    for (int dk = 0; dk < nk; dk++)
      for (int dj = 0; dj < nj; dj++)
        for (int di = 0; di < ni; di++) {
          const int64_t n = node_index(i0 + di, j0 + dj, k0 + dk, cx, cy);
          const double w = wi * wj * wk;
          for (int c = 0; c < 3; c++) acc[c] += w * ec[3 * n + c];
        }
    const unsigned b = bc_f[q];
    for (int c = 0; c < 3; c++)
      if (!((b >> c) & 1u)) xf[3 * q + c] += acc[c];
  }
}

// Coarse node I takes v and the Dirichlet bits of fine node 2I.
__global__ void inject_kernel(const double* __restrict__ vf, const uint8_t* __restrict__ bcf,
                              int fx, int fy, double* __restrict__ vc, uint8_t* __restrict__ bcc,
                              int cx, int cy, int cz) {
  const int64_t Nc = (int64_t)cx * cy * cz;
  GRID_STRIDE(q, Nc) {
    const int I = (int)(q % cx), J = (int)((q / cx) % cy), K = (int)(q / ((int64_t)cx * cy));
    const int64_t n = node_index(2 * I, 2 * J, 2 * K, fx, fy);
    vc[q] = vf[n];
    bcc[q] = bcf[n];
  }
}

// Coarse cell modulus = mean of its 8 children.
__global__ void cell_mean_kernel(const float* __restrict__ ef, int fcx, int fcy,
                                 float* __restrict__ ec, int ccx, int ccy, int ccz) {
  const int64_t Nc = (int64_t)ccx * ccy * ccz;
  GRID_STRIDE(q, Nc) {
    const int I = (int)(q % ccx), J = (int)((q / ccx) % ccy), K = (int)(q / ((int64_t)ccx * ccy));
    float s = 0.f;
    for (int dk = 0; dk < 2; dk++)
      for (int dj = 0; dj < 2; dj++)
        for (int di = 0; di < 2; di++)
          s += ef[((int64_t)(2 * K + dk) * fcy + (2 * J + dj)) * fcx + (2 * I + di)];
    ec[q] = 0.125f * s;
  }
}

// r = dinv * (b - t), or dinv * b when t is null (x = 0); d = r / theta.
__global__ void cheb_init_kernel(const double* __restrict__ b, const double* __restrict__ t,
                                 const double* __restrict__ dinv, double* __restrict__ r,
                                 double* __restrict__ d, double inv_theta, int64_t n) {
  GRID_STRIDE(i, n) {
    const double ri = dinv[i] * (t ? b[i] - t[i] : b[i]);
    r[i] = ri;
    d[i] = ri * inv_theta;
  }
}

// x += d; and unless last: r -= dinv * t (t = A d); d = c1 d + c2 r.
__global__ void cheb_step_kernel(double* __restrict__ x, double* __restrict__ d,
                                 double* __restrict__ r, const double* __restrict__ t,
                                 const double* __restrict__ dinv, double c1, double c2, int last,
                                 int64_t n) {
  GRID_STRIDE(i, n) {
    const double di = d[i];
    x[i] += di;
    if (!last) {
      const double ri = r[i] - dinv[i] * t[i];
      r[i] = ri;
      d[i] = c1 * di + c2 * ri;
    }
  }
}

// Deterministic start vector of the power iteration (0 on Dirichlet dofs).
__global__ void seed_kernel(double* __restrict__ x, const uint8_t* __restrict__ bc, int64_t N) {
  GRID_STRIDE(q, N) {
    const unsigned b = bc[q];
    for (int c = 0; c < 3; c++) {
      const uint64_t h = (uint64_t)(3 * q + c) * 0x9E3779B97F4A7C15ull;
      x[3 * q + c] = ((b >> c) & 1u) ? 0. : (double)((h >> 11) & 0xFFFFF) / 1048576.0 - 0.5;
    }
  }
}

// y = dinv * t
__global__ void scale_kernel(const double* __restrict__ t, const double* __restrict__ dinv,
                             double* __restrict__ y, int64_t n) {
  GRID_STRIDE(i, n) y[i] = dinv[i] * t[i];
}

}  // namespace

// ---------------------------------------------------------------------------------
// The level's view as a U operator: apply, the element arguments for its diagonal.
struct LevelView {
  int nx, ny, nz;
  double hx, hy, hz;
  const TilePlan* plan;
  double* seam;
  const double* v;
  const uint8_t* bc;
  const uint8_t* elayer;
  const float* cellE;
  const ETab* tab;
  const double* dinv;
  const uint32_t* cflag;  // fine level under NOCOMPRESSION: the Jacobian's bits
};

static LevelView view(vfgpu_ctx* c, int l, const double* dinv0) {
  if (l == 0)
    return {c->nx, c->ny, c->nz, c->hx, c->hy, c->hz, &c->plan64, c->seam64,
            c->f[VFGPU_FIELD_V], c->bcU_bits, c->d_elayer, c->d_cellE, c->d_tab, dinv0,
            c->unilateral ? c->d_cflag : nullptr};
  const auto& L = c->mg[l];
  return {L.nx, L.ny, L.nz, L.hx, L.hy, L.hz, &L.plan, L.seam, L.v, L.bc, L.elayer, L.cellE,
          L.tab, L.dinv, nullptr};
}

static cudaError_t level_apply(vfgpu_ctx* c, const LevelView& V, const double* x, double* y) {
  UApplyArgs<double> A{};
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
  A.ihx = 1.0 / V.hx;
  A.ihy = 1.0 / V.hy;
  A.ihz = 1.0 / V.hz;
  A.vol = V.hx * V.hy * V.hz;
  A.eta = c->vf.eta;
  A.P = c->d_params;
  A.cflag = V.cflag;
  return launch_u_apply<double>(A, *V.plan, c->layers, c->stream);
}

static int64_t level_n3(vfgpu_ctx* c, int l) { return 3 * (l == 0 ? c->N : c->mg[l].N); }

void free_mg(vfgpu_ctx* c) {
  for (auto& L : c->mg) {
    void* bufs[] = {L.seam, L.v, L.dinv, L.x, L.b, L.r, L.d, L.t, L.bc, L.elayer, L.cellE, L.tab};
    for (void* p : bufs) cudaFree(p);
  }
  c->mg.clear();
  cudaFree(c->mg_z);
  c->mg_z = nullptr;
}

// Allocates the hierarchy (once per ctx).
static int mg_build(vfgpu_ctx* c) {
  if (!c->mg.empty()) return VFGPU_OK;
  c->mg.emplace_back();  // level 0: fine work vectors
  cudaError_t e = cudaSuccess;
  auto& L0 = c->mg[0];
  const size_t n3 = 3 * (size_t)c->N * sizeof(double);
  for (double** p : {&L0.x, &L0.r, &L0.d, &L0.t, &c->mg_z})
    if (e == cudaSuccess) e = cudaMalloc((void**)p, n3);
  int nx = c->nx, ny = c->ny, nz = c->nz;
  double hx = c->hx, hy = c->hy, hz = c->hz;
  while (e == cudaSuccess && (nx - 1) % 2 == 0 && (ny - 1) % 2 == 0 && (nz - 1) % 2 == 0 &&
         (nx - 1) / 2 + 1 >= 5 && (ny - 1) / 2 + 1 >= 5 && (nz - 1) / 2 + 1 >= 5) {
    nx = (nx - 1) / 2 + 1;
    ny = (ny - 1) / 2 + 1;
    nz = (nz - 1) / 2 + 1;
    hx *= 2;
    hy *= 2;
    hz *= 2;
    vfgpu_ctx::MGLevel L;
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.N = (int64_t)nx * ny * nz;
    L.NC = (int64_t)(nx - 1) * (ny - 1) * (nz - 1);
    L.hx = hx;
    L.hy = hy;
    L.hz = hz;
    L.plan = u_plan(nx, ny, nz, 8, c->nsm);
    const size_t b3 = 3 * (size_t)L.N * sizeof(double);
    if (e == cudaSuccess)
      e = cudaMalloc((void**)&L.seam, std::max<size_t>(1, L.plan.seamX + L.plan.seamY) * sizeof(double));
    for (double** p : {&L.dinv, &L.x, &L.b, &L.r, &L.d, &L.t})
      if (e == cudaSuccess) e = cudaMalloc((void**)p, b3);
    if (e == cudaSuccess) e = cudaMalloc((void**)&L.v, L.N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&L.bc, L.N);
    if (e == cudaSuccess) e = cudaMalloc((void**)&L.elayer, nz - 1);
    if (e == cudaSuccess && c->d_cellE) e = cudaMalloc((void**)&L.cellE, L.NC * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&L.tab, sizeof(ETab));
    if (e == cudaSuccess) {
      ETab t;
      etab_host(hx, hy, hz, &t);
      e = cudaMemcpyAsync(L.tab, &t, sizeof t, cudaMemcpyHostToDevice, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
    c->mg.push_back(L);
  }
  if (e != cudaSuccess || c->mg.size() < 2) {
    free_mg(c);
    if (e != cudaSuccess) return cuda_fail(e, "multigrid hierarchy");
    return fail(VFGPU_ERR_INVALID,
                "multigrid needs an even cell count on every axis and >= 9 nodes per axis");
  }
  return VFGPU_OK;
}

// Per solve: coarse fields from the fine ones, diagonals, lmax per level.
static int mg_setup(vfgpu_ctx* c, const double* dinv0) {
  cudaError_t e = cudaSuccess;
  // coarse modulus buffers follow the ctx (set_cell_modulus may have added one)
  for (size_t l = 1; l < c->mg.size() && e == cudaSuccess; l++) {
    auto& L = c->mg[l];
    if (c->d_cellE && !L.cellE) e = cudaMalloc((void**)&L.cellE, L.NC * sizeof(float));
  }
  std::vector<uint8_t> el(std::max(1, c->nz - 1));
  if (e == cudaSuccess) e = cudaMemcpyAsync(el.data(), c->d_elayer, el.size(), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  for (size_t l = 1; l < c->mg.size() && e == cudaSuccess; l++) {
    auto& L = c->mg[l];
    const LevelView F = view(c, (int)l - 1, dinv0);
    inject_kernel<<<blocks_for(L.N), 256, 0, c->stream>>>(F.v, F.bc, F.nx, F.ny, L.v, L.bc, L.nx,
                                                          L.ny, L.nz);
    e = cudaGetLastError();
    std::vector<uint8_t> lc(L.nz - 1);
    for (int k = 0; k < L.nz - 1; k++) lc[k] = el[(size_t)k << l];  // lower child layer
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.elayer, lc.data(), lc.size(), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // lc leaves scope
    if (e == cudaSuccess && c->d_cellE) {
      cell_mean_kernel<<<blocks_for(L.NC), 256, 0, c->stream>>>(F.cellE, F.nx - 1, F.ny - 1, L.cellE,
                                                               L.nx - 1, L.ny - 1, L.nz - 1);
      e = cudaGetLastError();
    }
    // diagonal of the level operator (t as scratch)
    if (e == cudaSuccess) {
      ElemArgs E{};
      E.tab = L.tab;
      E.nx = L.nx;
      E.ny = L.ny;
      E.nz = L.nz;
      E.elayer = L.elayer;
      E.cellE = c->d_cellE ? L.cellE : nullptr;
      E.L = c->layers;
      E.eta = c->vf.eta;
      e = launch_u_diag(E, L.v, L.bc, L.t, c->stream);
      if (e == cudaSuccess) e = dev_inv(L.t, L.dinv, nullptr, 3 * L.N, c->stream);
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "multigrid set-up");
  // largest eigenvalue of D^-1 K per level by power iteration
  for (size_t l = 0; l < c->mg.size(); l++) {
    const LevelView V = view(c, (int)l, dinv0);
    const int64_t n3 = level_n3(c, (int)l);
    double* x = c->mg[l].x;
    double* t = c->mg[l].t;
    double* y = c->mg[l].d;
    seed_kernel<<<blocks_for(n3 / 3), 256, 0, c->stream>>>(x, V.bc, n3 / 3);
    e = cudaGetLastError();
    double lam = 0.;
    for (int it = 0; it < kPowerIts && e == cudaSuccess; it++) {
      e = level_apply(c, V, x, t);
      if (e == cudaSuccess) {
        scale_kernel<<<blocks_for(n3), 256, 0, c->stream>>>(t, V.dinv, y, n3);
        e = cudaGetLastError();
      }
      const double* pa[2] = {y, x};
      const double* pb[2] = {y, x};
      if (e == cudaSuccess) e = dev_dots(pa, pb, 2, n3, c->d_red, c->d_out, c->stream);
      double h[2] = {0., 0.};
      if (e == cudaSuccess) e = cudaMemcpyAsync(h, c->d_out, sizeof h, cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess || !(h[0] > 0.) || !(h[1] > 0.)) break;
      lam = sqrt(h[0] / h[1]);
      // x = y / |y|
      e = cudaMemsetAsync(x, 0, n3 * sizeof(double), c->stream);
      if (e == cudaSuccess) e = dev_axpy(x, 1.0 / sqrt(h[0]), y, n3, c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(e, "multigrid eigenvalue estimate");
    if (!(lam > 0.)) return fail(VFGPU_ERR_STATE, "multigrid: no positive eigenvalue estimate of a level operator");
    c->mg[l].lmax = 1.1 * lam;
  }
  return VFGPU_OK;
}

// Chebyshev iteration on D^-1 K x = D^-1 b of degree deg on [lo lmax, lmax]; x is
// updated in place (zero_start: x = 0 on entry, so no initial residual apply).
static cudaError_t chebyshev(vfgpu_ctx* c, const LevelView& V, int l, const double* b, double* x,
                             int deg, double lo, bool zero_start) {
  auto& L = c->mg[l];
  const int64_t n3 = level_n3(c, l);
  const double lmax = L.lmax, lmin = lo * lmax;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  double rho = 1.0 / sigma;
  cudaError_t e = cudaSuccess;
  if (zero_start) {
    e = cudaMemsetAsync(x, 0, n3 * sizeof(double), c->stream);
  } else {
    e = level_apply(c, V, x, L.t);
  }
  if (e == cudaSuccess) {
    cheb_init_kernel<<<blocks_for(n3), 256, 0, c->stream>>>(b, zero_start ? nullptr : L.t, V.dinv,
                                                           L.r, L.d, 1.0 / theta, n3);
    e = cudaGetLastError();
  }
  for (int k = 0; k < deg && e == cudaSuccess; k++) {
    const bool last = k == deg - 1;
    double c1 = 0., c2 = 0.;
    if (!last) {
      e = level_apply(c, V, L.d, L.t);
      const double rho_new = 1.0 / (2.0 * sigma - rho);
      c1 = rho_new * rho;
      c2 = 2.0 * rho_new / delta;
      rho = rho_new;
    }
    if (e == cudaSuccess) {
      cheb_step_kernel<<<blocks_for(n3), 256, 0, c->stream>>>(x, L.d, L.r, L.t, V.dinv, c1, c2,
                                                             last ? 1 : 0, n3);
      e = cudaGetLastError();
    }
  }
  return e;
}

// z = V-cycle(b) at level l (z and b are the level's own vectors, or the fine ones).
static cudaError_t vcycle(vfgpu_ctx* c, int l, const double* dinv0, const double* b, double* z) {
  const LevelView V = view(c, l, dinv0);
  const int last = (int)c->mg.size() - 1;
  if (l == last) return chebyshev(c, V, l, b, z, kCoarseDeg, kCoarseLo, true);
  cudaError_t e = chebyshev(c, V, l, b, z, kSmoothDeg, kSmoothLo, true);
  auto& L = c->mg[l];
  auto& C = c->mg[l + 1];
  const int64_t n3 = level_n3(c, l);
  // residual b - K z into L.r (t = K z)
  if (e == cudaSuccess) e = level_apply(c, V, z, L.t);
  if (e == cudaSuccess) e = dev_axpby(L.r, b, -1.0, L.t, n3, c->stream);
  if (e == cudaSuccess) {
    restrict_kernel<<<blocks_for(C.N), 256, 0, c->stream>>>(L.r, V.bc, V.nx, V.ny, V.nz, C.b, C.nx,
                                                           C.ny, C.nz, C.bc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = vcycle(c, l + 1, dinv0, C.b, C.x);
  if (e == cudaSuccess) {
    prolong_add_kernel<<<blocks_for(n3 / 3), 256, 0, c->stream>>>(C.x, C.nx, C.ny, z, V.nx, V.ny,
                                                                 V.nz, V.bc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = chebyshev(c, V, l, b, z, kSmoothDeg, kSmoothLo, false);
  return e;
}

// PCG with the V-cycle as preconditioner.  Stopping test of the Jacobi-preconditioned
// solve it replaces (KSPCG's preconditioned norm with B = D^-1): ||D^-1 r|| <=
// max(rtol ||D^-1 b||, atol), diverged on ||D^-1 r|| >= dtol ||D^-1 b||, NaN, an
// indefinite p.Kp or maxit, so that both preconditioners stop at the same residual.
// Scalars are read back on the host once per iteration.
int run_mgcg(vfgpu_ctx* c, const double* b, double* x, double* r, double* p, double* w,
             const double* dinv0, double rtol, double atol, double dtol, int maxit, int* its,
             int* reason, int* levels) {
  int rc = mg_build(c);
  if (rc) return rc;
  rc = mg_setup(c, dinv0);
  if (rc) return rc;
  *levels = (int)c->mg.size();
  const int64_t n3 = 3 * c->N;
  double* z = c->mg_z;
  cudaError_t e = cudaMemsetAsync(x, 0, n3 * sizeof(double), c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(r, b, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  // out[0] = a0.b0, out[1] = a1.b1 (a1 null: skipped), out[2] = ||D^-1 r||^2
  double h[3] = {0., 0., 0.};
  auto scalars = [&](const double* a0, const double* b0, const double* a1, const double* b1) {
    const double* pa[2] = {a0, a1};
    const double* pb[2] = {b0, b1};
    if (e == cudaSuccess) e = dev_dots(pa, pb, a1 ? 2 : 1, n3, c->d_red, c->d_out, c->stream);
    if (e == cudaSuccess) e = dev_znorm2(r, dinv0, n3, c->d_red, c->d_out + 2, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, c->d_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  };
  if (e == cudaSuccess) e = vcycle(c, 0, dinv0, r, z);
  scalars(r, z, nullptr, nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "multigrid PCG");
  double rz = h[0];
  const double rnorm0 = sqrt(h[2]), ttol = std::max(rtol * rnorm0, atol);
  *its = 0;
  *reason = 0;
  if (!(rnorm0 == rnorm0)) *reason = CG_DIVERGED_NAN;
  else if (rnorm0 <= ttol) *reason = rnorm0 <= atol ? CG_CONVERGED_ATOL : CG_CONVERGED_RTOL;
  else if (!(rz > 0.)) *reason = rz == 0. ? CG_CONVERGED_ATOL : CG_DIVERGED_INDEFINITE;
  if (!*reason) e = cudaMemcpyAsync(p, z, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  while (!*reason && e == cudaSuccess) {
    e = level_apply(c, view(c, 0, dinv0), p, w);
    const double* pa[1] = {p};
    const double* pb[1] = {w};
    if (e == cudaSuccess) e = dev_dots(pa, pb, 1, n3, c->d_red, c->d_out, c->stream);
    double pw = 0.;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&pw, c->d_out, sizeof pw, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) break;
    if (!(pw > 0.)) {
      *reason = (pw == pw) ? CG_DIVERGED_INDEFINITE : CG_DIVERGED_NAN;
      break;
    }
    const double alpha = rz / pw;
    e = dev_axpy(x, alpha, p, n3, c->stream);
    if (e == cudaSuccess) e = dev_axpy(r, -alpha, w, n3, c->stream);
    if (e == cudaSuccess) e = vcycle(c, 0, dinv0, r, z);
    scalars(r, z, nullptr, nullptr);
    if (e != cudaSuccess) break;
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

}  // namespace vfgpu
