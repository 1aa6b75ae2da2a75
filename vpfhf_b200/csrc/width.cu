// width.cu -- the flow-coupling boundary on the device: the fracture width
// UpdateFractureWidth (VFPermfield.c:267-562), its cell-to-node average
// CellToNodeInterpolation (VFPermfield.c:1156-1330) and the fracture well rate
// VolumetricFractureWellRate (VFPermfield.c:1513-1604).
//
// Width: one thread per cell.  A cell whose centre value of V lies in (0, 1) marches
// from its centre along +n and then -n (n = grad V / |grad V|) in steps of
// len = |n (hx, hy, hz)| / 20, integrating grad V . U and grad V over each step,
// until the integration length, V >= 1 or a turn of the direction ends it.  The
// reference finds the cell of each point by scanning every cell and keeping the last
// whose closed box holds it; per axis that is the largest index i with
// X[i] <= c <= X[i+1], found here from floor(c / h) and its two neighbours with the
// same comparisons; a point in no cell keeps the previous point's cell, as the
// reference's loop variables do.  Points are evaluated with the reference's point
// element (CartFEElement3DInit, VFCartFE.c:1837-1866, whose 1-D map is
// var = (x - l/2)/l/2).  This file is compiled without FMA contraction and every
// expression keeps the reference's operation order, so the widths are the oracle's
// to the bit.  A band cell with zero grad V at its centre cannot advance (len = 0;
// the reference's march does not end there): it keeps width 0 and is counted.
#include <cmath>

#include "abi_util.h"
#include "solver.h"

namespace vfgpu {
namespace {

constexpr int kMaxSteps = 1 << 20;

struct WidthArgs {
  const double* __restrict__ u;
  const double* __restrict__ v;
  double* __restrict__ widthc;
  double* __restrict__ pmult;
  unsigned* __restrict__ nstall;
  int nx, ny, nz;
  double lx, ly, lz, L, tol;
  int remove_tip;
};

__device__ __forceinline__ double coord(int i, double l, int n) {
  return i == 0 ? 0. : i * l / (n - 1.);
}

struct PtElem {
  double phi[8], dphi[8][3];
};

__device__ void pt_basis1d(double x, double l, double phi[2], double dphi[2]) {
  const double var = (x - l / 2.) / l / 2.;
  phi[0] = (1. - var) * .5;
  phi[1] = (1. + var) * .5;
  dphi[0] = -1. / l;
  dphi[1] = 1. / l;
}

__device__ void pt_elem(double x, double y, double z, double lx, double ly, double lz, PtElem& s) {
  double px[2], py[2], pz[2], dx[2], dy[2], dz[2];
  pt_basis1d(x, lx, px, dx);
  pt_basis1d(y, ly, py, dy);
  pt_basis1d(z, lz, pz, dz);
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int a = i + 2 * j + 4 * k;
        s.phi[a] = pz[k] * py[j] * px[i];
        s.dphi[a][0] = pz[k] * py[j] * dx[i];
        s.dphi[a][1] = pz[k] * dy[j] * px[i];
        s.dphi[a][2] = dz[k] * py[j] * px[i];
      }
}

// ComputeAveVGradVandNormal_local (VFPermfield.c:2124-2156)
__device__ void pt_fields(const WidthArgs& A, int ei, int ej, int ek, const PtElem& s,
                          double& vave, double g[3], double n[3], double uc[3]) {
  vave = 0.;
  for (int c = 0; c < 3; c++) g[c] = n[c] = uc[c] = 0.;
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int a = i + 2 * j + 4 * k;
        const int64_t q = node_index(ei + i, ej + j, ek + k, A.nx, A.ny);
        const double vq = A.v[q];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          g[c] += vq * s.dphi[a][c];
          uc[c] += A.u[3 * q + c] * s.phi[a];
        }
        vave += vq * s.phi[a];
      }
  const double mag = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  for (int c = 0; c < 3; c++) n[c] = g[c] / mag;
  if (!isfinite(n[0]) || !isfinite(n[1]) || !isfinite(n[2])) n[0] = n[1] = n[2] = 0.;
}

// IntegrateUcdotGradVlocal (VFPermfield.c:589-610) on VFCartFEElement1DInit(len)
__device__ __forceinline__ void seg_integrate(double& acc, double f0, double f1, const double w[3],
                                              const double phi[2][3]) {
  double fe[3] = {0., 0., 0.};
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int g = 0; g < 3; g++) fe[g] += (i ? f1 : f0) * phi[i][g];
#pragma unroll
  for (int g = 0; g < 3; g++) acc += fe[g] * w[g] / 2.;
}

// Largest cell index i with X[i] <= c <= X[i+1], or -1.
__device__ int axis_cell(double c, double l, int n) {
  const int ncell = n - 1;
  int i0 = (int)floor(c / (l / (n - 1.)));
  i0 = i0 < 0 ? 0 : (i0 > ncell - 1 ? ncell - 1 : i0);
  for (int i = min(i0 + 1, ncell - 1); i >= max(i0 - 1, 0); i--)
    if (coord(i + 1, l, n) >= c && coord(i, l, n) <= c) return i;
  return -1;
}

__device__ void cell_h(const WidthArgs& A, int ei, int ej, int ek, double& hx, double& hy,
                       double& hz) {
  hx = coord(ei + 1, A.lx, A.nx) - coord(ei, A.lx, A.nx);
  hy = coord(ej + 1, A.ly, A.ny) - coord(ej, A.ly, A.ny);
  hz = coord(ek + 1, A.lz, A.nz) - coord(ek, A.lz, A.nz);
}

// One march from the centre of (ei,ej,ek) along dir * n; returns true if it hit the
// step cap.
__device__ bool march(const WidthArgs& A, int ei, int ej, int ek, int dir, double len, int cur[3],
                      double& w, double val[3]) {
  double hx, hy, hz, vave, g[3], n[3], uc[3], ref[3], g0[3], ca[3], cc[3];
  PtElem s;
  cell_h(A, ei, ej, ek, hx, hy, hz);
  pt_elem(hx / 2., hy / 2., hz / 2., hx, hy, hz, s);
  pt_fields(A, ei, ej, ek, s, vave, g, n, uc);
  for (int c = 0; c < 3; c++) {
    ref[c] = n[c];
    g0[c] = g[c];
  }
  double cod0 = g[0] * uc[0] + g[1] * uc[1] + g[2] * uc[2];
  ca[0] = (coord(ei + 1, A.lx, A.nx) + coord(ei, A.lx, A.nx)) / 2.;
  ca[1] = (coord(ej + 1, A.ly, A.ny) + coord(ej, A.ly, A.ny)) / 2.;
  ca[2] = (coord(ek + 1, A.lz, A.nz) + coord(ek, A.lz, A.nz)) / 2.;
  for (int c = 0; c < 3; c++) cc[c] = dir > 0 ? ca[c] + n[c] * len : ca[c] - n[c] * len;
  // VFCartFEElement1DInit(len) (VFCartFE.c:90-116): Gauss weights and basis values
  const double r35 = sqrt(3. / 5.);
  const double sw[3] = {5. * len / 18., 8. * len / 18., 5. * len / 18.};
  const double sphi[2][3] = {{(1. + r35) * .5, .5, (1. - r35) * .5},
                             {(1. - r35) * .5, .5, (1. + r35) * .5}};
  double lc = len;
  int steps = 0;
  do {
    const int fi = axis_cell(cc[0], A.lx, A.nx), fj = axis_cell(cc[1], A.ly, A.ny),
              fk = axis_cell(cc[2], A.lz, A.nz);
    if (fi >= 0 && fj >= 0 && fk >= 0) {
      cur[0] = fi;
      cur[1] = fj;
      cur[2] = fk;
    }
    cell_h(A, cur[0], cur[1], cur[2], hx, hy, hz);
    const double hwx = cc[0] - coord(cur[0], A.lx, A.nx);
    const double hwy = cc[1] - coord(cur[1], A.ly, A.ny);
    const double hwz = cc[2] - coord(cur[2], A.lz, A.nz);
    const double nold[3] = {n[0], n[1], n[2]};
    pt_elem(hwx, hwy, hwz, hx, hy, hz, s);
    pt_fields(A, cur[0], cur[1], cur[2], s, vave, g, n, uc);
    const double cod1 = g[0] * uc[0] + g[1] * uc[1] + g[2] * uc[2];
    seg_integrate(w, cod0, cod1, sw, sphi);
    for (int c = 0; c < 3; c++) seg_integrate(val[c], g0[c], g[c], sw, sphi);
    if (n[0] == 0 && n[1] == 0 && n[2] == 0)
      for (int c = 0; c < 3; c++) n[c] = nold[c];
    double c1[3], c2[3];
    for (int c = 0; c < 3; c++) {
      c1[c] = cc[c] + n[c] * len;
      c2[c] = cc[c] - n[c] * len;
    }
    const double t1 = sqrt((c1[0] - ca[0]) * (c1[0] - ca[0]) + (c1[1] - ca[1]) * (c1[1] - ca[1]) +
                           (c1[2] - ca[2]) * (c1[2] - ca[2]));
    const double t2 = sqrt((c2[0] - ca[0]) * (c2[0] - ca[0]) + (c2[1] - ca[1]) * (c2[1] - ca[1]) +
                           (c2[2] - ca[2]) * (c2[2] - ca[2]));
    if (t1 > t2) {
      for (int c = 0; c < 3; c++) cc[c] = c1[c];
    } else {
      for (int c = 0; c < 3; c++) {
        cc[c] = c2[c];
        n[c] = -1 * n[c];
      }
    }
    lc += len;
    cod0 = cod1;
    for (int c = 0; c < 3; c++) g0[c] = g[c];
    if (++steps >= kMaxSteps) return true;
  } while (lc < A.L - len && vave < 1.0 &&
           (dir > 0 ? ref[0] * n[0] + ref[1] * n[1] + ref[2] * n[2] >= 0.
                    : -ref[0] * n[0] - ref[1] * n[1] - ref[2] * n[2] >= 0.));
  return false;
}

__global__ void __launch_bounds__(128) width_kernel(const WidthArgs A) {
  const int64_t ncell = (int64_t)(A.nx - 1) * (A.ny - 1) * (A.nz - 1);
  for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < ncell;
       cell += (int64_t)gridDim.x * blockDim.x) {
    const int ei = (int)(cell % (A.nx - 1));
    const int ej = (int)((cell / (A.nx - 1)) % (A.ny - 1));
    const int ek = (int)(cell / ((int64_t)(A.nx - 1) * (A.ny - 1)));
    double hx, hy, hz, vave, g[3], n[3], uc[3], w = 0., val[3] = {0., 0., 0.}, value = 0.;
    PtElem s;
    cell_h(A, ei, ej, ek, hx, hy, hz);
    pt_elem(hx / 2., hy / 2., hz / 2., hx, hy, hz, s);
    pt_fields(A, ei, ej, ek, s, vave, g, n, uc);
    const double len =
        sqrt((n[0] * hx) * (n[0] * hx) + (n[1] * hy) * (n[1] * hy) + (n[2] * hz) * (n[2] * hz)) / 20;
    double pm = 1.;
    if (vave < 1.0 && vave > 0.0) {
      if (!(len > 0.)) {
        atomicAdd(A.nstall, 1u);
      } else {
        int cur[3] = {ei, ej, ek};
        const bool s1 = march(A, ei, ej, ek, 1, len, cur, w, val);
        const bool s2 = march(A, ei, ej, ek, -1, len, cur, w, val);
        if (s1 || s2) atomicAdd(A.nstall, 1u);
        value = sqrt(val[0] * val[0] + val[1] * val[1] + val[2] * val[2]);
        if (value > A.tol) pm = 0.;
      }
    }
    if (w < 0.0) w = 0;
    if (A.remove_tip && value > A.tol) w = 0;
    A.widthc[cell] = w;
    A.pmult[cell] = pm;
  }
}

// Node = sum over its cells (ascending cell order) of w h^3 / sum of h^3.
__global__ void cell_to_node_kernel(const double* __restrict__ cellv, double* __restrict__ nodev,
                                    int nx, int ny, int nz, double lx, double ly, double lz) {
  const int64_t N = (int64_t)nx * ny * nz;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((int64_t)nx * ny));
    double vol = 0., acc = 0.;
    for (int ek = max(k - 1, 0); ek <= min(k, nz - 2); ek++)
      for (int ej = max(j - 1, 0); ej <= min(j, ny - 2); ej++)
        for (int ei = max(i - 1, 0); ei <= min(i, nx - 2); ei++) {
          const double hx = coord(ei + 1, lx, nx) - coord(ei, lx, nx);
          const double hy = coord(ej + 1, ly, ny) - coord(ej, ly, ny);
          const double hz = coord(ek + 1, lz, nz) - coord(ek, lz, nz);
          vol += hz * hy * hx;
          acc += cellv[((int64_t)ek * (ny - 1) + ej) * (nx - 1) + ei] * hx * hy * hz;
        }
    nodev[q] = acc / vol;
  }
}

constexpr int kRateThreads = 256, kRateBlocks = 592;

// Block partials of sum over cells of sum_g regrate(g) |grad V(g)| w_g (VFPermfield.c:1513-1549).
__global__ void __launch_bounds__(kRateThreads)
    well_rate_kernel(const __grid_constant__ ETab tab, const double* __restrict__ v,
                     const double* __restrict__ r, int nx, int ny, int nz,
                     double* __restrict__ partial) {
  __shared__ double scratch[32];
  const int64_t ncell = (int64_t)(nx - 1) * (ny - 1) * (nz - 1);
  double acc = 0.;
  for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < ncell;
       cell += (int64_t)gridDim.x * blockDim.x) {
    const int ei = (int)(cell % (nx - 1));
    const int ej = (int)((cell / (nx - 1)) % (ny - 1));
    const int ek = (int)(cell / ((int64_t)(nx - 1) * (ny - 1)));
    double v8[8], r8[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
      const int64_t q = node_index(ei + (a & 1), ej + ((a >> 1) & 1), ek + (a >> 2), nx, ny);
      v8[a] = v[q];
      r8[a] = r[q];
    }
    double loc = 0.;
    for (int g = 0; g < 27; g++) {
      double d0 = 0., d1 = 0., d2 = 0., rg = 0.;
#pragma unroll
      for (int a = 0; a < 8; a++) {
        d0 += v8[a] * tab.dphi[a][0][g];
        d1 += v8[a] * tab.dphi[a][1][g];
        d2 += v8[a] * tab.dphi[a][2][g];
        rg += r8[a] * tab.phi[a][g];
      }
      loc += rg * sqrt(d0 * d0 + d1 * d1 + d2 * d2) * tab.w[g];
    }
    acc += loc;
  }
  const double b = block_sum_dbl(acc, scratch);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

__global__ void rate_final_kernel(const double* __restrict__ partial, int nb, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.;
    for (int b = 0; b < nb; b++) s += partial[b];
    out[0] = s;
  }
}

// WidthIntLenght (VFCommon.c:897-914)
double width_int_length(const vfgpu_ctx* c) {
  const double bx = c->lx / (c->nx - 1), by = c->ly / (c->ny - 1), bz = c->lz / (c->nz - 1);
  double res;
  if (c->nx == 2) res = by < bz ? by : bz;
  else if (c->ny == 2) res = bx < bz ? bx : bz;
  else if (c->nz == 2) res = bx < by ? bx : by;
  else if (bx < by && bx < bz) res = bx;
  else if (by < bx && by < bz) res = by;
  else res = bz;
  return 3 * res + 4 * c->vf.epsilon;
}

int width_buffers(vfgpu_ctx* c) {
  if (c->d_widthc) return VFGPU_OK;
  cudaError_t e = cudaMalloc((void**)&c->d_widthc, std::max<int64_t>(1, c->NC) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_pmult, std::max<int64_t>(1, c->NC) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_width, c->N * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_wstall, sizeof(unsigned));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&c->d_wpart, (c->N + c->NC + kRateBlocks + 1) * sizeof(double));
  if (e != cudaSuccess) {
    for (void* p : {(void*)c->d_widthc, (void*)c->d_pmult, (void*)c->d_width, (void*)c->d_wstall,
                    (void*)c->d_wpart})
      cudaFree(p);
    c->d_widthc = c->d_pmult = c->d_width = c->d_wpart = nullptr;
    c->d_wstall = nullptr;
    return cuda_fail(e, "fracture width buffers");
  }
  return VFGPU_OK;
}

}  // namespace
}  // namespace vfgpu

using namespace vfgpu;

extern "C" {

void vfgpu_default_width_opts(vfgpu_width_opts* o) {
  if (!o) return;
  o->int_length = 0.;       // 3 res + 4 epsilon at the call
  o->width_tol = 0.1;       // VFCommon.c:111
  o->remove_tip_effect = 0; // VFCommon.c:108
}

int vfgpu_update_fracture_width(vfgpu_ctx* c, const vfgpu_width_opts* o_, double* widthc,
                                double* width, double* pmult, int* nstalled) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_update_fracture_width: null ctx");
  vfgpu_width_opts o;
  if (o_) o = *o_; else vfgpu_default_width_opts(&o);
  if (!(o.width_tol == o.width_tol) || !(o.int_length == o.int_length))
    return fail(VFGPU_ERR_INVALID, "vfgpu_update_fracture_width: NaN option");
  cudaSetDevice(c->dev);
  int rc = width_buffers(c);
  if (rc) return rc;
  WidthArgs A{};
  A.u = c->f[VFGPU_FIELD_U];
  A.v = c->f[VFGPU_FIELD_V];
  A.widthc = c->d_widthc;
  A.pmult = c->d_pmult;
  A.nstall = c->d_wstall;
  A.nx = c->nx;
  A.ny = c->ny;
  A.nz = c->nz;
  A.lx = c->lx;
  A.ly = c->ly;
  A.lz = c->lz;
  A.L = o.int_length > 0 ? o.int_length : width_int_length(c);
  A.tol = o.width_tol;
  A.remove_tip = o.remove_tip_effect != 0;
  cudaError_t e = cudaMemsetAsync(c->d_wstall, 0, sizeof(unsigned), c->stream);
  const int blocks = (int)std::min<int64_t>((c->NC + 127) / 128, (int64_t)c->nsm * 16);
  if (e == cudaSuccess && c->NC > 0) {
    width_kernel<<<blocks, 128, 0, c->stream>>>(A);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    cell_to_node_kernel<<<(int)std::min<int64_t>((c->N + 255) / 256, (int64_t)c->nsm * 16), 256, 0,
                          c->stream>>>(c->d_widthc, c->d_width, c->nx, c->ny, c->nz, c->lx, c->ly,
                                       c->lz);
    e = cudaGetLastError();
  }
  unsigned stall = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&stall, c->d_wstall, sizeof stall, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && widthc) e = copy_out(c, widthc, c->d_widthc, c->NC);
  if (e == cudaSuccess && width) e = copy_out(c, width, c->d_width, c->N);
  if (e == cudaSuccess && pmult) e = copy_out(c, pmult, c->d_pmult, c->NC);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_update_fracture_width");
  if (nstalled) *nstalled = (int)stall;
  return VFGPU_OK;
}

int vfgpu_cell_to_node(vfgpu_ctx* c, const double* cellv, double* nodev) {
  if (!c || !cellv || !nodev) return fail(VFGPU_ERR_INVALID, "vfgpu_cell_to_node: null argument");
  cudaSetDevice(c->dev);
  int rc = width_buffers(c);
  if (rc) return rc;
  // d_wpart: the node values (N), then the cell values (NC)
  double* nd = c->d_wpart;
  double* cd = c->d_wpart + c->N;
  cudaError_t e = copy_in(c, cd, cellv, c->NC);
  if (e == cudaSuccess) {
    cell_to_node_kernel<<<(int)std::min<int64_t>((c->N + 255) / 256, (int64_t)c->nsm * 16), 256, 0,
                          c->stream>>>(cd, nd, c->nx, c->ny, c->nz, c->lx, c->ly, c->lz);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = copy_out(c, nodev, nd, c->N);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_cell_to_node");
  return VFGPU_OK;
}

int vfgpu_fracture_well_rate(vfgpu_ctx* c, const double* regrate, double* rate) {
  if (!c || !regrate || !rate) return fail(VFGPU_ERR_INVALID, "vfgpu_fracture_well_rate: null argument");
  cudaSetDevice(c->dev);
  int rc = width_buffers(c);
  if (rc) return rc;
  // d_wpart: the nodal rate (N), (NC unused), the block partials, the sum
  double* r = c->d_wpart;
  double* partial = c->d_wpart + c->N + c->NC;
  double* out = partial + kRateBlocks;
  cudaError_t e = copy_in(c, r, regrate, c->N);
  if (e == cudaSuccess) {
    ETab t;
    etab_host(c->hx, c->hy, c->hz, &t);
    well_rate_kernel<<<kRateBlocks, kRateThreads, 0, c->stream>>>(t, c->f[VFGPU_FIELD_V], r, c->nx,
                                                                 c->ny, c->nz, partial);
    rate_final_kernel<<<1, 32, 0, c->stream>>>(partial, kRateBlocks, out);
    e = cudaGetLastError();
  }
  double h = 0.;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) *rate = h;
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_fracture_well_rate");
  return VFGPU_OK;
}

}  // extern "C"
