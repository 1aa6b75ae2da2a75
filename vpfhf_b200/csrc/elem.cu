// elem.cu -- once-per-solve element kernels, written per Gauss point after the
// reference's element routines.  Scatter to nodes is done in 8 parity colours of
// elements so that no two threads of a launch touch the same node: deterministic, no
// atomics.  The element tables travel by value in the kernel parameters
// (__grid_constant__): every thread of a warp reads the same entry, which the
// constant bank broadcasts.
#include <cmath>

#include "elem.h"

namespace vfgpu {

void etab_host(double hx, double hy, double hz, ETab* e) {
  // VFCartFEElement1DInit (VFCartFE.c:90-116), tensor product as VFCartFEElement3DInit.
  auto t1 = [](double l, double w[3], double phi[2][3], double dphi[2][3]) {
    w[0] = 5. * l / 18.;
    w[1] = 8. * l / 18.;
    w[2] = 5. * l / 18.;
    phi[0][0] = (1. + sqrt(3. / 5.)) * .5;
    phi[0][1] = .5;
    phi[0][2] = (1. - sqrt(3. / 5.)) * .5;
    phi[1][0] = (1. - sqrt(3. / 5.)) * .5;
    phi[1][1] = .5;
    phi[1][2] = (1. + sqrt(3. / 5.)) * .5;
    for (int g = 0; g < 3; g++) {
      dphi[0][g] = -1. / l;
      dphi[1][g] = 1. / l;
    }
  };
  double wx[3], wy[3], wz[3], px[2][3], py[2][3], pz[2][3], dx[2][3], dy[2][3], dz[2][3];
  t1(hx, wx, px, dx);
  t1(hy, wy, py, dy);
  t1(hz, wz, pz, dz);
  for (int gk = 0, g = 0; gk < 3; gk++)
    for (int gj = 0; gj < 3; gj++)
      for (int gi = 0; gi < 3; gi++, g++) {
        e->w[g] = wz[gk] * wy[gj] * wx[gi];
        for (int k = 0; k < 2; k++)
          for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
              const int a = i + 2 * j + 4 * k;
              e->phi[a][g] = pz[k][gk] * py[j][gj] * px[i][gi];
              e->dphi[a][0][g] = pz[k][gk] * py[j][gj] * dx[i][gi];
              e->dphi[a][1][g] = pz[k][gk] * dy[j][gj] * px[i][gi];
              e->dphi[a][2][g] = dz[k][gk] * py[j][gj] * px[i][gi];
            }
      }
}

namespace {

struct CellMat {
  double lambda, mu, alpha, beta, Gc;
};

__device__ __forceinline__ CellMat cell_mat(const ElemArgs& E, int ei, int ej, int ek) {
  const int l = E.elayer ? E.elayer[ek] : 0;
  CellMat m;
  if (E.cellE) {
    const double Ec = (double)E.cellE[((int64_t)ek * (E.ny - 1) + ej) * (E.nx - 1) + ei];
    m.lambda = Ec * E.L.lamfac[l];
    m.mu = Ec * E.L.mufac[l];
  } else {
    m.lambda = E.L.lambda[l];
    m.mu = E.L.mu[l];
  }
  m.alpha = E.L.alpha[l];
  m.beta = E.L.beta[l];
  m.Gc = E.L.Gc[l];
  return m;
}

__device__ __forceinline__ void cell_nodes(const ElemArgs& E, int ei, int ej, int ek,
                                           int64_t (&n)[8]) {
#pragma unroll
  for (int a = 0; a < 8; a++)
    n[a] = node_index(ei + (a & 1), ej + ((a >> 1) & 1), ek + (a >> 2), E.nx, E.ny);
}

// Element (ei,ej,ek) of colour (cx,cy,cz) for the linear thread index t, or false.
__device__ __forceinline__ bool colour_cell(const ElemArgs& E, int color, int64_t t, int& ei,
                                            int& ej, int& ek) {
  const int cx = color & 1, cy = (color >> 1) & 1, cz = color >> 2;
  const int hx = (E.nx - 1 - cx + 1) / 2, hy = (E.ny - 1 - cy + 1) / 2, hz = (E.nz - 1 - cz + 1) / 2;
  if (t >= (int64_t)hx * hy * hz) return false;
  ei = cx + 2 * (int)(t % hx);
  ej = cy + 2 * (int)((t / hx) % hy);
  ek = cz + 2 * (int)(t / ((int64_t)hx * hy));
  return true;
}

// tr(eps(u)) at Gauss point g from the 8 nodal displacements, in the reference's order
__device__ __forceinline__ double trace_at(const ETab& e, const double (&u8)[8][3], int g) {
  double tr = 0.;
  for (int a = 0; a < 8; a++)
    tr += e.dphi[a][0][g] * u8[a][0] + e.dphi[a][1][g] * u8[a][1] + e.dphi[a][2][g] * u8[a][2];
  return tr;
}

__device__ __forceinline__ void gather_u8(const int64_t (&n)[8], const double* __restrict__ u,
                                          double (&u8)[8][3]) {
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++) u8[a][c] = u ? u[3 * n[a] + c] : 0.;
}

// ---- tensor-product forms (the plain operator).  On the uniform grid the 27-point rule
// is the tensor product of the 1-D rule, and every table entry is a product of 1-D
// factors: phi_a(g) = b_k(gz) b_j(gy) b_i(gx), dphi_a,x(g) = b_k(gz) b_j(gy) (-+1/hx),
// w_g = W_gx W_gy W_gz vol, with b_0(g) = (1 + sqrt(3/5))/2, 1/2, (1 - sqrt(3/5))/2 at
// the three points, b_1 the mirror, W = 5/18, 8/18, 5/18 (VFCartFEElement1DInit,
// VFCartFE.c:90-116).  So fields at the points, the integrals against products of
// basis functions and the scatter back to the nodes are each three 1-D passes.
constexpr double kB0 = 0.5 * (1.0 + 0.774596669241483377035853079956);  // (1 + sqrt(3/5))/2
constexpr double kB2 = 0.5 * (1.0 - 0.774596669241483377035853079956);
__device__ __forceinline__ constexpr double bas(int i, int g) {
  return g == 1 ? 0.5 : ((g == 0) == (i == 0) ? kB0 : kB2);
}
__device__ __forceinline__ constexpr double w1(int g) { return g == 1 ? 8.0 / 18.0 : 5.0 / 18.0; }

// Modal form of a trilinear field on the unit cell t in [-1/2, 1/2]^3: f = sum_p m_p t^p
// (p = px + 2 py + 4 pz; m_0 the mean, m_1 the x slope, ...), and its value and
// gradient at the Gauss point (gx, gy, gz), t = -tau, 0, +tau.  With the point
// indices known at compile time (unrolled loops) each is a short chain of FMAs, and
// the compiler shares the partial sums between points.
__device__ __forceinline__ void modal_of(const double (&f)[8], double (&m)[8]) {
  double a[8], b[8];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    a[2 * p] = 0.5 * (f[2 * p] + f[2 * p + 1]);
    a[2 * p + 1] = f[2 * p + 1] - f[2 * p];
  }
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int al = 0; al < 2; al++) {
      const double lo = a[al + 4 * k], hi = a[al + 2 + 4 * k];
      b[al + 4 * k] = 0.5 * (lo + hi);
      b[al + 2 + 4 * k] = hi - lo;
    }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const double lo = b[q], hi = b[q + 4];
    m[q] = 0.5 * (lo + hi);
    m[q + 4] = hi - lo;
  }
}
__device__ __forceinline__ double mlin(int g, double a, double b) {
  return g == 1 ? a : (g == 0 ? fma(b, -VF_TAU, a) : fma(b, VF_TAU, a));
}
__device__ __forceinline__ double mval(const double (&m)[8], int gx, int gy, int gz) {
  return mlin(gz, mlin(gy, mlin(gx, m[0], m[1]), mlin(gx, m[2], m[3])),
              mlin(gy, mlin(gx, m[4], m[5]), mlin(gx, m[6], m[7])));
}
__device__ __forceinline__ double mdx(const double (&m)[8], int gx, int gy, int gz, double ih) {
  return ih * mlin(gy, mlin(gz, m[1], m[5]), mlin(gz, m[3], m[7]));
}
__device__ __forceinline__ double mdy(const double (&m)[8], int gx, int gy, int gz, double ih) {
  return ih * mlin(gx, mlin(gz, m[2], m[6]), mlin(gz, m[3], m[7]));
}
__device__ __forceinline__ double mdz(const double (&m)[8], int gx, int gy, int gz, double ih) {
  return ih * mlin(gx, mlin(gy, m[4], m[6]), mlin(gy, m[5], m[7]));
}

// Trilinear field at the 27 points, g = gx + 3 gy + 9 gz.
__device__ __forceinline__ void interp27(const double (&f)[8], double (&o)[27]) {
  double fx[4][3], fy[2][3][3];
#pragma unroll
  for (int jk = 0; jk < 4; jk++)
#pragma unroll
    for (int g = 0; g < 3; g++) fx[jk][g] = bas(0, g) * f[2 * jk] + bas(1, g) * f[2 * jk + 1];
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int gy = 0; gy < 3; gy++)
#pragma unroll
      for (int gx = 0; gx < 3; gx++)
        fy[k][gy][gx] = bas(0, gy) * fx[2 * k][gx] + bas(1, gy) * fx[2 * k + 1][gx];
#pragma unroll
  for (int gz = 0; gz < 3; gz++)
#pragma unroll
    for (int gy = 0; gy < 3; gy++)
#pragma unroll
      for (int gx = 0; gx < 3; gx++)
        o[gx + 3 * gy + 9 * gz] = bas(0, gz) * fy[0][gy][gx] + bas(1, gz) * fy[1][gy][gx];
}

// out[i + 2j + 4k] = sum_g q_g b_i(gx) b_j(gy) b_k(gz)
__device__ __forceinline__ void contract27(const double (&q)[27], double (&out)[8]) {
  double cx[2][3][3], cy[2][2][3];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int gz = 0; gz < 3; gz++)
#pragma unroll
      for (int gy = 0; gy < 3; gy++) {
        const int b = 3 * gy + 9 * gz;
        cx[i][gy][gz] = (bas(i, 0) * q[b] + bas(i, 1) * q[b + 1]) + bas(i, 2) * q[b + 2];
      }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int gz = 0; gz < 3; gz++)
        cy[i][j][gz] = (bas(j, 0) * cx[i][0][gz] + bas(j, 1) * cx[i][1][gz]) + bas(j, 2) * cx[i][2][gz];
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++)
        out[i + 2 * j + 4 * k] =
            (bas(k, 0) * cy[i][j][0] + bas(k, 1) * cy[i][j][1]) + bas(k, 2) * cy[i][j][2];
}

// out[i + 2j + 4k] = sum_g q_g b_i(gx)^2 b_j(gy)^2 b_k(gz)^2
__device__ __forceinline__ void contract27sq(const double (&q)[27], double (&out)[8]) {
  auto f = [](int p, int g) { return bas(p, g) * bas(p, g); };
  double cx[2][3][3], cy[2][2][3];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int gz = 0; gz < 3; gz++)
#pragma unroll
      for (int gy = 0; gy < 3; gy++) {
        const int b = 3 * gy + 9 * gz;
        cx[i][gy][gz] = (f(i, 0) * q[b] + f(i, 1) * q[b + 1]) + f(i, 2) * q[b + 2];
      }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int gz = 0; gz < 3; gz++)
        cy[i][j][gz] = (f(j, 0) * cx[i][0][gz] + f(j, 1) * cx[i][1][gz]) + f(j, 2) * cx[i][2][gz];
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++)
        out[i + 2 * j + 4 * k] = (f(k, 0) * cy[i][j][0] + f(k, 1) * cy[i][j][1]) + f(k, 2) * cy[i][j][2];
}

// Integrals of q against the squared or plain basis products that carry no factor
// along axis d: F[d][p][q] = sum_g q_g f_p(g_e1) f_q(g_e2) with (e1, e2) the other two
// axes in increasing order, f = b (SQ = false) or b^2 (SQ = true).
template <bool SQ>
__device__ __forceinline__ void face_moments(const double (&q)[27], double (&F)[3][2][2]) {
  auto f = [](int p, int g) { return SQ ? bas(p, g) * bas(p, g) : bas(p, g); };
  double R[3][3][3];  // R[d][ga][gb]: q summed along axis d, indexed by the other two
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      R[0][a][b] = (q[0 + 3 * a + 9 * b] + q[1 + 3 * a + 9 * b]) + q[2 + 3 * a + 9 * b];  // (gy, gz)
      R[1][a][b] = (q[a + 0 + 9 * b] + q[a + 3 + 9 * b]) + q[a + 6 + 9 * b];              // (gx, gz)
      R[2][a][b] = (q[a + 3 * b] + q[a + 3 * b + 9]) + q[a + 3 * b + 18];                 // (gx, gy)
    }
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int pq = 0; pq < 2; pq++) {
      double t[3];
#pragma unroll
      for (int a = 0; a < 3; a++) t[a] = (f(pq, 0) * R[d][a][0] + f(pq, 1) * R[d][a][1]) + f(pq, 2) * R[d][a][2];
#pragma unroll
      for (int p = 0; p < 2; p++) F[d][p][pq] = (f(p, 0) * t[0] + f(p, 1) * t[1]) + f(p, 2) * t[2];
    }
}

// u_diag_kernel in tensor form (plain operator): diag of node (i,j,k), component x, is
//   (lambda + 2 mu) Jx[j][k] / hx^2 + mu (Jy[i][k] / hy^2 + Jz[i][j] / hz^2)
// with J_d the integrals of w (v^2 + eta) against the squared basis functions of the
// other two axes (and similarly for y, z).
__global__ void u_diag_tp_kernel(const __grid_constant__ ElemArgs E, int color,
                                 const double* __restrict__ v, double* __restrict__ d) {
  int ei, ej, ek;
  if (!colour_cell(E, color, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  double v8[8], v27[27], s27[27];
#pragma unroll
  for (int a = 0; a < 8; a++) v8[a] = v[n[a]];
  interp27(v8, v27);
  const double vol = E.hx * E.hy * E.hz;
#pragma unroll
  for (int gz = 0; gz < 3; gz++)
#pragma unroll
    for (int gy = 0; gy < 3; gy++)
#pragma unroll
      for (int gx = 0; gx < 3; gx++) {
        const int g = gx + 3 * gy + 9 * gz;
        s27[g] = (vol * (w1(gx) * w1(gy) * w1(gz))) * fma(v27[g], v27[g], E.eta);
      }
  double J[3][2][2];
  face_moments<true>(s27, J);
  const CellMat m = cell_mat(E, ei, ej, ek);
  const double l2m = m.lambda + 2. * m.mu;
  const double ih2[3] = {1. / (E.hx * E.hx), 1. / (E.hy * E.hy), 1. / (E.hz * E.hz)};
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const double jx = J[0][j][k] * ih2[0], jy = J[1][i][k] * ih2[1], jz = J[2][i][j] * ih2[2];
        const int64_t q = 3 * n[i + 2 * j + 4 * k];
        d[q + 0] += fma(l2m, jx, m.mu * (jy + jz));
        d[q + 1] += fma(l2m, jy, m.mu * (jx + jz));
        d[q + 2] += fma(l2m, jz, m.mu * (jx + jy));
      }
}

// u_rhs_kernel in tensor form (plain operator): the thermo-poro load
// sum_g w dphi_a,c S_g, S = 3 kappa alpha (theta - thetaRef)(v^2 + eta) + beta p v, as
// face moments of w S times -+1/h_c, and the crack-pressure load
// sum_g w p grad_c v phi_a as a full contraction.
__global__ void u_rhs_tp_kernel(const __grid_constant__ ElemArgs E, int color,
                                const double* __restrict__ v, const double* __restrict__ theta,
                                const double* __restrict__ thetaRef, const double* __restrict__ p,
                                double* __restrict__ f) {
  int ei, ej, ek;
  if (!colour_cell(E, color, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  double v8[8], th8[8], p8[8];
#pragma unroll
  for (int a = 0; a < 8; a++) {
    v8[a] = v[n[a]];
    th8[a] = theta ? theta[n[a]] - (thetaRef ? thetaRef[n[a]] : 0.) : 0.;
    p8[a] = p ? p[n[a]] : 0.;
  }
  const CellMat m = cell_mat(E, ei, ej, ek);
  const double coefalpha = (3. * m.lambda + 2. * m.mu) * m.alpha, beta = m.beta;
  const double vol = E.hx * E.hy * E.hz;
  double ve[27], pe[27], ws[27];
  interp27(v8, ve);
  interp27(p8, pe);
  {
    double te[27];
    interp27(th8, te);
#pragma unroll
    for (int gz = 0; gz < 3; gz++)
#pragma unroll
      for (int gy = 0; gy < 3; gy++)
#pragma unroll
        for (int gx = 0; gx < 3; gx++) {
          const int g = gx + 3 * gy + 9 * gz;
          const double s = coefalpha * te[g] * (ve[g] * ve[g] + E.eta) + beta * pe[g] * ve[g];
          ws[g] = (vol * (w1(gx) * w1(gy) * w1(gz))) * s;
        }
  }
  double F[3][2][2];
  face_moments<false>(ws, F);
  const double ih[3] = {1. / E.hx, 1. / E.hy, 1. / E.hz};
  double rl[8][3];
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int a = i + 2 * j + 4 * k;
        rl[a][0] = (i ? ih[0] : -ih[0]) * F[0][j][k];
        rl[a][1] = (j ? ih[1] : -ih[1]) * F[1][i][k];
        rl[a][2] = (k ? ih[2] : -ih[2]) * F[2][i][j];
      }
  if (E.hasCrackPressure) {
    // grad v at the points: each component depends on the two other axes only
    double gv[3][9];  // gv[d][a + 3 b], (a, b) the other axes' point indices
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) {
        double sx = 0., sy = 0., sz = 0.;
#pragma unroll
        for (int q = 0; q < 2; q++)
#pragma unroll
          for (int r = 0; r < 2; r++) {
            sx += bas(q, a) * bas(r, b) * (v8[1 + 2 * q + 4 * r] - v8[2 * q + 4 * r]);
            sy += bas(q, a) * bas(r, b) * (v8[q + 2 + 4 * r] - v8[q + 4 * r]);
            sz += bas(q, a) * bas(r, b) * (v8[q + 2 * r + 4] - v8[q + 2 * r]);
          }
        gv[0][a + 3 * b] = sx * ih[0];
        gv[1][a + 3 * b] = sy * ih[1];
        gv[2][a + 3 * b] = sz * ih[2];
      }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double qc[27], oc[8];
#pragma unroll
      for (int gz = 0; gz < 3; gz++)
#pragma unroll
        for (int gy = 0; gy < 3; gy++)
#pragma unroll
          for (int gx = 0; gx < 3; gx++) {
            const int g = gx + 3 * gy + 9 * gz;
            const double gvc = c == 0 ? gv[0][gy + 3 * gz] : (c == 1 ? gv[1][gx + 3 * gz] : gv[2][gx + 3 * gy]);
            qc[g] = (vol * (w1(gx) * w1(gy) * w1(gz))) * pe[g] * gvc;
          }
      contract27(qc, oc);
#pragma unroll
      for (int a = 0; a < 8; a++) rl[a][c] += oc[a];
    }
  }
#pragma unroll
  for (int a = 0; a < 8; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) f[3 * n[a] + c] += rl[a][c];
}

__global__ void u_rhs_kernel(const __grid_constant__ ElemArgs E, int color, const double* __restrict__ v,
                             const double* __restrict__ theta, const double* __restrict__ thetaRef,
                             const double* __restrict__ p, double* __restrict__ f,
                             const double* __restrict__ u0) {
  int ei, ej, ek;
  if (!colour_cell(E, color, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  const ETab& e = E.tab;
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  double v8[8], th8[8], p8[8], rl[24];
#pragma unroll
  for (int a = 0; a < 8; a++) {
    v8[a] = v[n[a]];
    th8[a] = theta ? theta[n[a]] - (thetaRef ? thetaRef[n[a]] : 0.) : 0.;
    p8[a] = p ? p[n[a]] : 0.;
  }
  for (int l = 0; l < 24; l++) rl[l] = 0.;
  const CellMat m = cell_mat(E, ei, ej, ek);
  // VF_GradientUThermoPoro3D_local (VFMech.c:386-447); NOCOMPRESSION
  // (VFMech.c:456-524): undegraded thermal term and p instead of p v where tr < 0
  const double coefalpha = (3. * m.lambda + 2. * m.mu) * m.alpha, beta = m.beta;
  double u8[8][3];
  if (E.unilateral) gather_u8(n, u0, u8);
  for (int g = 0; g < 27; g++) {
    double te = 0., pe = 0., ve = 0.;
    for (int a = 0; a < 8; a++) {
      te += e.phi[a][g] * th8[a];
      pe += e.phi[a][g] * p8[a];
      ve += e.phi[a][g] * v8[a];
    }
    const bool comp = E.unilateral && trace_at(e, u8, g) < 0.;
    const double s = comp ? coefalpha * te * (1. + E.eta) + beta * pe
                          : coefalpha * te * (ve * ve + E.eta) + beta * pe * ve;
    for (int a = 0; a < 8; a++)
      for (int c = 0; c < 3; c++) rl[3 * a + c] += e.w[g] * e.dphi[a][c][g] * s;
  }
  // VF_GradientUCrackPressure3D_local (VFMech.c:533-589)
  if (E.hasCrackPressure) {
    for (int g = 0; g < 27; g++) {
      double pe = 0., gv[3] = {0., 0., 0.};
      for (int a = 0; a < 8; a++) {
        pe += e.phi[a][g] * p8[a];
        for (int c = 0; c < 3; c++) gv[c] += e.dphi[a][c][g] * v8[a];
      }
      for (int a = 0; a < 8; a++)
        for (int c = 0; c < 3; c++) rl[3 * a + c] += e.w[g] * pe * gv[c] * e.phi[a][g];
    }
  }
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++) f[3 * n[a] + c] += rl[3 * a + c];
}

__global__ void u_diag_kernel(const __grid_constant__ ElemArgs E, int color, const double* __restrict__ v,
                              double* __restrict__ d, const double* __restrict__ u0) {
  int ei, ej, ek;
  if (!colour_cell(E, color, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  const ETab& e = E.tab;
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  double v8[8], dg[24];
#pragma unroll
  for (int a = 0; a < 8; a++) v8[a] = v[n[a]];
  for (int l = 0; l < 24; l++) dg[l] = 0.;
  const CellMat m = cell_mat(E, ei, ej, ek);
  double u8[8][3];
  if (E.unilateral) gather_u8(n, u0, u8);
  const double kappa = m.lambda + 2. * m.mu / 3.;
  for (int g = 0; g < 27; g++) {
    double s = 0.;
    for (int a = 0; a < 8; a++) s += v8[a] * e.phi[a][g];
    const double sv = s * s + E.eta, ws = e.w[g] * sv;
    // spherical coefficient: lambda s, or kappa (1 + eta) - 2 mu s / 3 in compression
    const bool comp = E.unilateral && trace_at(e, u8, g) < 0.;
    const double lw = comp ? e.w[g] * (kappa * (1. + E.eta) - 2. * m.mu * sv / 3.) : ws * m.lambda;
    for (int a = 0; a < 8; a++) {
      const double d0 = e.dphi[a][0][g], d1 = e.dphi[a][1][g], d2 = e.dphi[a][2][g];
      const double g2 = d0 * d0 + d1 * d1 + d2 * d2;
      dg[3 * a + 0] += (lw + ws * m.mu) * d0 * d0 + ws * m.mu * g2;
      dg[3 * a + 1] += (lw + ws * m.mu) * d1 * d1 + ws * m.mu * g2;
      dg[3 * a + 2] += (lw + ws * m.mu) * d2 * d2 + ws * m.mu * g2;
    }
  }
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++) d[3 * n[a] + c] += dg[3 * a + c];
}

__global__ void nc_flags_kernel(const __grid_constant__ ElemArgs E, const double* __restrict__ u,
                                uint32_t* __restrict__ flags) {
  const int64_t NCELL = (int64_t)(E.nx - 1) * (E.ny - 1) * (E.nz - 1);
  const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= NCELL) return;
  const int ei = (int)(cell % (E.nx - 1));
  const int ej = (int)((cell / (E.nx - 1)) % (E.ny - 1));
  const int ek = (int)(cell / ((int64_t)(E.nx - 1) * (E.ny - 1)));
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  double u8[8][3];
  gather_u8(n, u, u8);
  uint32_t bits = 0u;
  for (int g = 0; g < 27; g++)
    if (trace_at(E.tab, u8, g) < 0.) bits |= 1u << g;
  flags[cell] = bits;
}

__global__ void bc_diag_kernel(const uint8_t* __restrict__ bcbits, double* __restrict__ d, int64_t N) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned b = bcbits[i];
    for (int c = 0; c < 3; c++)
      if ((b >> c) & 1u) d[3 * i + c] = 1.;
  }
}

// ElasticEnergyDensity3D_local (VFMech.c:32-106) at every Gauss point, times 2 and
// the Gauss weight, plus the AT2 mass coefficient (VFMech.c:2040-2058).  The strain at
// the points comes from the modal form of u (the same trilinear interpolant the
// reference's basis-function sums evaluate).
__global__ void __launch_bounds__(128) v_coef_kernel(const __grid_constant__ ElemArgs E,
                                                     const double* __restrict__ u,
                                                     const double* __restrict__ theta,
                                                     const double* __restrict__ thetaRef,
                                                     double* __restrict__ coef,
                                                     float* __restrict__ coef32) {
  const int64_t NCELL = (int64_t)(E.nx - 1) * (E.ny - 1) * (E.nz - 1);
  const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= NCELL) return;
  const int ei = (int)(cell % (E.nx - 1));
  const int ej = (int)((cell / (E.nx - 1)) % (E.ny - 1));
  const int ek = (int)(cell / ((int64_t)(E.nx - 1) * (E.ny - 1)));
  const int pitch = vcoef_pitch(E.nx - 1);
  const ETab& e = E.tab;
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  double mu3[3][8], mth[8];
  {
    double f[3][8], th8[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
#pragma unroll
      for (int c = 0; c < 3; c++) f[c][a] = u[3 * n[a] + c];
      th8[a] = theta ? theta[n[a]] - (thetaRef ? thetaRef[n[a]] : 0.) : 0.;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) modal_of(f[c], mu3[c]);
    modal_of(th8, mth);
  }
  const double ihx = 1. / E.hx, ihy = 1. / E.hy, ihz = 1. / E.hz;
  const CellMat m = cell_mat(E, ei, ej, ek);
  const double mass = E.atnum == 2 ? m.Gc / E.atcv * .5 / E.epsilon : 0.;
  const double l = m.lambda, mu = m.mu;
#pragma unroll
  for (int gz = 0; gz < 3; gz++)
#pragma unroll
    for (int gy = 0; gy < 3; gy++)
#pragma unroll
      for (int gx = 0; gx < 3; gx++) {
        const int g = gx + 3 * gy + 9 * gz;
        const double uxx = mdx(mu3[0], gx, gy, gz, ihx), uyy = mdy(mu3[1], gx, gy, gz, ihy);
        const double uzz = mdz(mu3[2], gx, gy, gz, ihz);
        const double e12 = (mdx(mu3[1], gx, gy, gz, ihx) + mdy(mu3[0], gx, gy, gz, ihy)) * .5;
        const double e23 = (mdy(mu3[2], gx, gy, gz, ihy) + mdz(mu3[1], gx, gy, gz, ihz)) * .5;
        const double e13 = (mdx(mu3[2], gx, gy, gz, ihx) + mdz(mu3[0], gx, gy, gz, ihz)) * .5;
        const double at = m.alpha * mval(mth, gx, gy, gz);
        double cgv;
        if (E.unilateral) {
          // ElasticEnergyDensitySphericalDeviatoricNoCompression3D_local (VFMech.c:115-218):
          // W = sigma(eps - e0) : eps, less (kappa/2) tr^2 where tr < 0
          const double kappa = l + 2. * mu / 3.;
          const double s11 = (l + 2. * mu) * (uxx - at) + l * (uyy - at) + l * (uzz - at);
          const double s22 = l * (uxx - at) + (l + 2. * mu) * (uyy - at) + l * (uzz - at);
          const double s33 = l * (uxx - at) + l * (uyy - at) + (l + 2. * mu) * (uzz - at);
          const double Wf = (s11 * uxx + s22 * uyy + s33 * uzz) * .5 +
                            2. * mu * (e12 * e12 + e23 * e23 + e13 * e13);
          const double tr = uxx + uyy + uzz;
          const double S = tr < 0. ? 0. : kappa * tr * tr * .5, D = Wf - kappa * tr * tr * .5;
          cgv = e.w[g] * (2. * (S + D) + mass);
        } else {
          const double e11 = uxx - at, e22 = uyy - at, e33 = uzz - at;
          const double s11 = (l + 2. * mu) * e11 + l * e22 + l * e33;
          const double s22 = l * e11 + (l + 2. * mu) * e22 + l * e33;
          const double s33 = l * e11 + l * e22 + (l + 2. * mu) * e33;
          const double W = (s11 * e11 + s22 * e22 + s33 * e33) * .5 +
                           2. * mu * (e12 * e12 + e23 * e23 + e13 * e13);
          cgv = e.w[g] * (2. * W + mass);
        }
        const int64_t ci = vcoef_index(g, ei, ej, ek, pitch, E.ny - 1);
        coef[ci] = cgv;
        if (coef32) coef32[ci] = (float)cgv;
      }
}


// V load (VF_ResidualVAT1/AT23D_local and VF_ResidualVCrackPressure3D_local,
// VFMech.c:2294-2384) in tensor form: the AT term coef sum_g w phi_a = coef vol / 8 per
// node, the crack-pressure term sum_g w p (u . grad phi_a) as face moments of w p u_c.
__global__ void v_rhs_tp_kernel(const __grid_constant__ ElemArgs E, int color,
                                const double* __restrict__ u, const double* __restrict__ p,
                                double* __restrict__ b) {
  int ei, ej, ek;
  if (!colour_cell(E, color, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  const CellMat m = cell_mat(E, ei, ej, ek);
  const double vol = E.hx * E.hy * E.hz;
  const double coef = m.Gc / E.atcv / E.epsilon * (E.atnum == 1 ? .25 : .5);
  double rl[8];
#pragma unroll
  for (int a = 0; a < 8; a++) rl[a] = coef * vol * 0.125;
  if (E.hasCrackPressure && p) {
    double p8[8], pe[27];
#pragma unroll
    for (int a = 0; a < 8; a++) p8[a] = p[n[a]];
    interp27(p8, pe);
    const double ih[3] = {1. / E.hx, 1. / E.hy, 1. / E.hz};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double u8[8], q[27], F[3][2][2];
#pragma unroll
      for (int a = 0; a < 8; a++) u8[a] = u[3 * n[a] + c];
      interp27(u8, q);
#pragma unroll
      for (int gz = 0; gz < 3; gz++)
#pragma unroll
        for (int gy = 0; gy < 3; gy++)
#pragma unroll
          for (int gx = 0; gx < 3; gx++) {
            const int g = gx + 3 * gy + 9 * gz;
            q[g] = (vol * (w1(gx) * w1(gy) * w1(gz))) * pe[g] * q[g];
          }
      face_moments<false>(q, F);
#pragma unroll
      for (int k = 0; k < 2; k++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
          for (int i = 0; i < 2; i++) {
            const int sgn = c == 0 ? i : (c == 1 ? j : k);
            const double fm = c == 0 ? F[0][j][k] : (c == 1 ? F[1][i][k] : F[2][i][j]);
            rl[i + 2 * j + 4 * k] += (sgn ? ih[c] : -ih[c]) * fm;
          }
    }
  }
#pragma unroll
  for (int a = 0; a < 8; a++) b[n[a]] += rl[a];
}

// Diagonal of K_V (the AT forms VF_BilinearFormVAT1/AT23D_local, VFMech.c:2040-2090,
// plus the coupling VF_BilinearFormVCoupling3D_local, :2093-2122) in tensor form:
// aeps sum_g w |grad phi_a|^2 from the face moments of w, plus sum_g coef_g phi_a^2 as
// a contraction against the squared basis.
__global__ void v_diag_tp_kernel(const __grid_constant__ ElemArgs E, int color,
                                 const double* __restrict__ coef, double* __restrict__ d) {
  int ei, ej, ek;
  if (!colour_cell(E, color, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  int64_t n[8];
  cell_nodes(E, ei, ej, ek, n);
  const CellMat m = cell_mat(E, ei, ej, ek);
  const double aeps = m.Gc / E.atcv * .5 * E.epsilon;
  const double vol = E.hx * E.hy * E.hz;
  const int pitch = vcoef_pitch(E.nx - 1);
  double w27[27], c27[27], J[3][2][2], M[8];
#pragma unroll
  for (int gz = 0; gz < 3; gz++)
#pragma unroll
    for (int gy = 0; gy < 3; gy++)
#pragma unroll
      for (int gx = 0; gx < 3; gx++) {
        const int g = gx + 3 * gy + 9 * gz;
        w27[g] = vol * (w1(gx) * w1(gy) * w1(gz));
        c27[g] = coef[vcoef_index(g, ei, ej, ek, pitch, E.ny - 1)];
      }
  face_moments<true>(w27, J);
  contract27sq(c27, M);
  const double ih2[3] = {1. / (E.hx * E.hx), 1. / (E.hy * E.hy), 1. / (E.hz * E.hz)};
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const double lap = (J[0][j][k] * ih2[0] + J[1][i][k] * ih2[1]) + J[2][i][j] * ih2[2];
        d[n[i + 2 * j + 4 * k]] += fma(aeps, lap, M[i + 2 * j + 4 * k]);
      }
}

// Neumaier-compensated accumulation.
struct KSum {
  double s = 0., c = 0.;
  __device__ void add(double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ double value() const { return s + c; }
};

constexpr int EN_THREADS = 128, EN_BLOCKS = 888;  // 6 blocks per SM of 148

// Value and gradient of a modal form (modal_of) at the point t = (tx, ty, tz).
__device__ __forceinline__ double mval_t(const double (&m)[8], double tx, double ty, double tz) {
  return fma(fma(fma(m[7], tx, m[6]), ty, fma(m[5], tx, m[4])), tz,
             fma(fma(m[3], tx, m[2]), ty, fma(m[1], tx, m[0])));
}
__device__ __forceinline__ double mdx_t(const double (&m)[8], double ty, double tz, double ih) {
  return ih * fma(fma(m[7], tz, m[3]), ty, fma(m[5], tz, m[1]));
}
__device__ __forceinline__ double mdy_t(const double (&m)[8], double tx, double tz, double ih) {
  return ih * fma(fma(m[7], tz, m[3]), tx, fma(m[6], tz, m[2]));
}
__device__ __forceinline__ double mdz_t(const double (&m)[8], double tx, double ty, double ih) {
  return ih * fma(fma(m[7], ty, m[5]), tx, fma(m[6], ty, m[4]));
}

// One thread per element (grid-stride, fixed assignment), per-thread compensated
// sums, pairwise tree in shared memory, per-block partials: deterministic.  The fields
// at the 27 points come from their modal forms (the trilinear interpolants the
// reference's basis-function sums evaluate); the point loop is not unrolled, which
// keeps the thread at < 170 registers (3 blocks per SM).
__global__ void __launch_bounds__(EN_THREADS, 3) energy_kernel(
    const __grid_constant__ ElemArgs E, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ theta, const double* __restrict__ thetaRef,
    const double* __restrict__ p, double* __restrict__ partial, double* __restrict__ cellcov) {
  __shared__ double red[4][EN_THREADS];
  const int64_t NCELL = (int64_t)(E.nx - 1) * (E.ny - 1) * (E.nz - 1);
  const double ihx = 1. / E.hx, ihy = 1. / E.hy, ihz = 1. / E.hz;
  const double vol = E.hx * E.hy * E.hz;
  KSum acc[4];
  for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < NCELL;
       cell += (int64_t)gridDim.x * blockDim.x) {
    const int ei = (int)(cell % (E.nx - 1));
    const int ej = (int)((cell / (E.nx - 1)) % (E.ny - 1));
    const int ek = (int)(cell / ((int64_t)(E.nx - 1) * (E.ny - 1)));
    int64_t n[8];
    cell_nodes(E, ei, ej, ek, n);
    const CellMat m = cell_mat(E, ei, ej, ek);
    double mu3[3][8], mv[8], mp[8], mth[8];
    {
      double f[3][8], v8[8], th8[8], p8[8];
#pragma unroll
      for (int a = 0; a < 8; a++) {
#pragma unroll
        for (int c = 0; c < 3; c++) f[c][a] = u[3 * n[a] + c];
        v8[a] = v[n[a]];
        th8[a] = theta ? theta[n[a]] - (thetaRef ? thetaRef[n[a]] : 0.) : 0.;
        p8[a] = p ? p[n[a]] : 0.;
      }
#pragma unroll
      for (int c = 0; c < 3; c++) modal_of(f[c], mu3[c]);
      modal_of(v8, mv);
      modal_of(p8, mp);
      modal_of(th8, mth);
    }
    const double threekappa = 3. * m.lambda + 2. * m.mu, coefbeta = m.beta / threekappa;
    const double scoef = m.Gc / E.atcv * .25;
    double el = 0., pw = 0., se = 0., cv = 0., wsum = 0.;
#pragma unroll 1
    for (int g = 0; g < 27; g++) {
      const int gx = g % 3, gy = (g / 3) % 3, gz = g / 9;
      const double tx = gx == 1 ? 0. : (gx == 0 ? -VF_TAU : VF_TAU);
      const double ty = gy == 1 ? 0. : (gy == 0 ? -VF_TAU : VF_TAU);
      const double tz = gz == 1 ? 0. : (gz == 0 ? -VF_TAU : VF_TAU);
      const double w = vol * (w1(gx) * w1(gy) * w1(gz));
      double D11 = mdx_t(mu3[0], ty, tz, ihx), D22 = mdy_t(mu3[1], tx, tz, ihy);
      double D33 = mdz_t(mu3[2], tx, ty, ihz);
      const double D12 = (mdx_t(mu3[1], ty, tz, ihx) + mdy_t(mu3[0], tx, tz, ihy)) * .5;
      const double D23 = (mdy_t(mu3[2], tx, tz, ihy) + mdz_t(mu3[1], tx, ty, ihz)) * .5;
      const double D13 = (mdx_t(mu3[2], ty, tz, ihx) + mdz_t(mu3[0], tx, ty, ihz)) * .5;
      const double ve = mval_t(mv, tx, ty, tz), pe = mval_t(mp, tx, ty, tz);
      const double te = mval_t(mth, tx, ty, tz);
      const double gv0 = mdx_t(mv, ty, tz, ihx), gv1 = mdy_t(mv, tx, tz, ihy), gv2 = mdz_t(mv, tx, ty, ihz);
      // VF_ElasticEnergy3D_local (VFMech.c:725-809), quirk Q2: v^2 (1+eta) on the deviator
      const double tr = D11 + D22 + D33;
      D11 -= tr / 3.;
      D22 -= tr / 3.;
      D33 -= tr / 3.;
      el += (D11 * D11 + D22 * D22 + D33 * D33 + (D12 * D12 + D23 * D23 + D13 * D13) * 2.) * ve * ve *
            (1. + E.eta) * m.mu * w;
      // NOCOMPRESSION (VF_ElasticEnergyNoCompression3D_local, VFMech.c:819-908): the
      // spherical factor is 1 instead of v where tr < 0
      const double sph = (E.unilateral && tr < 0.) ? 1. : ve;
      const double WD = (tr / 3. - m.alpha * te) * sph - coefbeta * pe;
      el += 3. * threekappa / 2. * WD * WD * w;
      el += threekappa / 6. * tr * tr * E.eta * w;
      const double udv = mval_t(mu3[0], tx, ty, tz) * gv0 + mval_t(mu3[1], tx, ty, tz) * gv1 +
                         mval_t(mu3[2], tx, ty, tz) * gv2;
      // VF_PressureWork3D_local (VFMech.c:920-974)
      if (E.hasCrackPressure) pw += w * pe * udv;
      // VF_AT1/AT2SurfaceEnergy3D_local (VFMech.c:2394-2465)
      const double g2 = gv0 * gv0 + gv1 * gv1 + gv2 * gv2;
      const double om = 1. - ve;
      se += w * ((E.atnum == 1 ? om : om * om) / E.epsilon + g2 * E.epsilon) * scoef;
      // VolumetricCrackOpening3D_local (VFPermfield.c:15-73)
      cv += udv * w;
      wsum += w;
    }
    if (cellcov) cellcov[cell] = cv / wsum;
    acc[0].add(el);
    acc[1].add(pw);
    acc[2].add(se);
    acc[3].add(cv);
  }
  for (int q = 0; q < 4; q++) red[q][threadIdx.x] = acc[q].value();
  __syncthreads();
  for (int st = EN_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 4; q++) red[q][threadIdx.x] += red[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 4) partial[blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void energy_final_kernel(const double* __restrict__ partial, int nblocks,
                                    double* __restrict__ out) {
  if (threadIdx.x >= 4) return;
  KSum s;
  for (int b = 0; b < nblocks; b++) s.add(partial[b * 4 + threadIdx.x]);
  out[threadIdx.x] = s.value();
}

template <typename K, typename... Args>
cudaError_t colours(const ElemArgs& E, K kernel, cudaStream_t s, Args... args) {
  for (int color = 0; color < 8; color++) {
    const int cx = color & 1, cy = (color >> 1) & 1, cz = color >> 2;
    const int64_t cnt = (int64_t)((E.nx - 1 - cx + 1) / 2) * ((E.ny - 1 - cy + 1) / 2) *
                        ((E.nz - 1 - cz + 1) / 2);
    if (cnt == 0) continue;
    kernel<<<(int)((cnt + 127) / 128), 128, 0, s>>>(E, color, args...);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_u_rhs(const ElemArgs& E, const double* v, const double* theta,
                         const double* thetaRef, const double* p, double* f, cudaStream_t s,
                         const double* u0) {
  const int64_t N = (int64_t)E.nx * E.ny * E.nz;
  cudaError_t e = cudaMemsetAsync(f, 0, 3 * N * sizeof(double), s);
  if (e != cudaSuccess) return e;
  if (!E.unilateral) return colours(E, u_rhs_tp_kernel, s, v, theta, thetaRef, p, f);
  return colours(E, u_rhs_kernel, s, v, theta, thetaRef, p, f, u0);
}

cudaError_t launch_nc_flags(const ElemArgs& E, const double* u, uint32_t* flags, cudaStream_t s) {
  const int64_t NCELL = (int64_t)(E.nx - 1) * (E.ny - 1) * (E.nz - 1);
  nc_flags_kernel<<<(int)((NCELL + 127) / 128), 128, 0, s>>>(E, u, flags);
  return cudaGetLastError();
}

cudaError_t launch_u_diag(const ElemArgs& E, const double* v, const uint8_t* bcbits, double* d,
                          cudaStream_t s, const double* u0) {
  const int64_t N = (int64_t)E.nx * E.ny * E.nz;
  cudaError_t e = cudaMemsetAsync(d, 0, 3 * N * sizeof(double), s);
  if (e == cudaSuccess)
    e = E.unilateral ? colours(E, u_diag_kernel, s, v, d, u0) : colours(E, u_diag_tp_kernel, s, v, d);
  if (e == cudaSuccess && bcbits) {
    bc_diag_kernel<<<(int)std::min<int64_t>((N + 255) / 256, 2368), 256, 0, s>>>(bcbits, d, N);
    e = cudaGetLastError();
  }
  return e;
}

cudaError_t launch_v_coef(const ElemArgs& E, const double* u, const double* theta,
                          const double* thetaRef, double* coef, float* coef32, cudaStream_t s) {
  const int64_t NCELL = (int64_t)(E.nx - 1) * (E.ny - 1) * (E.nz - 1);
  v_coef_kernel<<<(int)((NCELL + 127) / 128), 128, 0, s>>>(E, u, theta, thetaRef, coef, coef32);
  return cudaGetLastError();
}

cudaError_t launch_v_rhs(const ElemArgs& E, const double* u, const double* p, double* b,
                         cudaStream_t s) {
  const int64_t N = (int64_t)E.nx * E.ny * E.nz;
  cudaError_t e = cudaMemsetAsync(b, 0, N * sizeof(double), s);
  if (e != cudaSuccess) return e;
  return colours(E, v_rhs_tp_kernel, s, u, p, b);
}

cudaError_t launch_v_diag(const ElemArgs& E, const double* coef, double* d, cudaStream_t s) {
  const int64_t N = (int64_t)E.nx * E.ny * E.nz;
  cudaError_t e = cudaMemsetAsync(d, 0, N * sizeof(double), s);
  if (e != cudaSuccess) return e;
  return colours(E, v_diag_tp_kernel, s, coef, d);
}

int energy_blocks() { return EN_BLOCKS; }

cudaError_t launch_energies(const ElemArgs& E, const double* u, const double* v,
                            const double* theta, const double* thetaRef, const double* p,
                            double* partial, double* out, double* cellcov, cudaStream_t s) {
  energy_kernel<<<EN_BLOCKS, EN_THREADS, 0, s>>>(E, u, v, theta, thetaRef, p, partial, cellcov);
  energy_final_kernel<<<1, 32, 0, s>>>(partial, EN_BLOCKS, out);
  return cudaGetLastError();
}

}  // namespace vfgpu
