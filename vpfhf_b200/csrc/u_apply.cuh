// u_apply.cuh -- matrix-free apply of the phase-field-degraded Q1-hex elasticity
// operator K(v) (VF_BilinearFormU3D_local, VFMech.c:227-290, applied as in
// VF_UResidual, VFMech.c:1555-1596) on sm_100a.
//
// Element math ("modal" sum factorisation).  On the uniform DMDA grid every
// element is the same box, so in local coordinates t in [-1/2,1/2]^3 a
// trilinear field is f(t) = sum_{abc} m_abc P_a(tx) P_b(ty) P_c(tz) with
// P_0 = 1, P_1 = t; the 8 modal coefficients come from 3 butterfly passes
// ((lo+hi)/2, hi-lo) over the nodal values.  Then
//   d/dx f = (1/hx) (m_100 + m_110 ty + m_101 tz + m_111 ty tz)
// does not depend on tx, and similarly for y and z, so the 3x3 gradient at the
// 27 Gauss points of the reference's rule (t = -tau, 0, tau, tau = sqrt(3/5)/2,
// weights 5/18, 8/18, 5/18) costs a few FMAs per point.  The stress
//   sigma = w (v^2 + eta) (lambda tr(G) I + mu (G + G^T))
// is accumulated into 4 bilinear moments per (component, direction), and the
// transpose y_(a,c) = sum_g sum_d dphi_a,d(g) sigma_cd(g) is rebuilt from those
// moments with the inverse butterfly.  About 1.4k operations per element,
// against 8,856 for the per-Gauss-point form and ~233k for the element-matrix
// form the reference uses.
//
// The schedule (tiles, z-march, seams) is in tile_engine.cuh, the operator
// policy in ops.cuh.
//
// Dirichlet rows (MatZeroRowsStencil, VFCartFE.c:1293, quirk: rows only): on a
// BC dof the output is y = x; BC columns are kept.
#pragma once

#include "common.cuh"

namespace vfgpu {

template <typename T> struct UApplyArgs {
  CUtensorMap xmap, vmap;             // 1-D tensor maps of x (3N) and v (N) for the operators that
                                      // copy node planes by tensor copies (Op::PLANES_TMA)
  const T* __restrict__ x;            // 3N interlaced input
  const T* __restrict__ v;            // N phase field
  T* __restrict__ y;                  // 3N output
  const uint8_t* __restrict__ bc;     // N: bit c => dof (node,c) is Dirichlet
  const uint8_t* __restrict__ elayer; // nz-1: material layer of element layer ek (or null)
  const float* __restrict__ cellE;    // per-cell Young's modulus (or null)
  T* __restrict__ seamX;              // x-seam partials [(ntx-1)][nz][ny][4][3]
  T* __restrict__ seamY;              // y-seam partials [(nty-1)][nz][nx][2][3]
  const int* __restrict__ skip;       // if non-null and *skip != 0 the launch does nothing
  const DevParams* __restrict__ P;    // material and eta; null => the by-value LayerTable and eta
  double* __restrict__ dot;           // if non-null: per-block partials of x.y (see tile_engine.cuh)
  const uint32_t* __restrict__ cflag; // NOCOMPRESSION: per cell, bit g = tr(eps(u0)) < 0 at Gauss
                                      // point g (u_element_nc); null = the plain operator
  // Unit lists (null ur[l]: the launch splits all (tile, node plane) units): list 0 holds
  // the units whose two adjacent element layers have a constant nodal v throughout the
  // tile (the fixed-weight operator UOpConst), list 1 the rest (UOp).  The launch's
  // blocks share the utotal[l] units of runs ur[l] (x: tile column, y: first plane, z: end
  // plane, w: units before the run) evenly; block b starts in run ustart[l][b].
  const int4* __restrict__ ur[2];
  const int* __restrict__ ustart[2];
  const int* __restrict__ utotal;
  unsigned* __restrict__ plane_err;   // set when a bounded wait on a plane copy gave up
  int nx, ny, nz;
  int ntx, nty;                       // tiles in x, y
  T ihx, ihy, ihz, vol, eta;
};

// Modal transform of nodal values f[a], a = i + 2j + 4k, into m[p], p = a + 2b + 4c
// with 0 = mean, 1 = difference along each axis.
template <typename T>
__device__ __forceinline__ void modal8(const T (&f)[8], T (&m)[8]) {
  T a[8], b[8];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    a[2 * p] = T(0.5) * (f[2 * p] + f[2 * p + 1]);
    a[2 * p + 1] = f[2 * p + 1] - f[2 * p];
  }
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int al = 0; al < 2; al++) {
      T lo = a[al + 4 * k], hi = a[al + 2 + 4 * k];
      b[al + 4 * k] = T(0.5) * (lo + hi);
      b[al + 2 + 4 * k] = hi - lo;
    }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    T lo = b[q], hi = b[q + 4];
    m[q] = T(0.5) * (lo + hi);
    m[q + 4] = hi - lo;
  }
}

// a + b*t_g for Gauss index g (t_1 = 0 is folded at compile time).
template <typename T> __device__ __forceinline__ T lin(int g, T a, T b) {
  return g == 1 ? a : (g == 0 ? fma(b, T(-VF_TAU), a) : fma(b, T(VF_TAU), a));
}
// Gauss weights and points as double constants (products of them fold at compile
// time before the conversion to T).
__device__ __forceinline__ constexpr double gwd(int g) { return g == 1 ? VF_W1 : VF_W0; }
__device__ __forceinline__ constexpr double gtd(int g) { return g == 1 ? 0.0 : (g == 0 ? -VF_TAU : VF_TAU); }
template <typename T> __device__ __forceinline__ T gw(int g) { return T(gwd(g)); }
template <typename T> __device__ __forceinline__ T gt(int g) { return T(gtd(g)); }

// Moment update q[0..3] += s * {1, t1, t2, t1 t2} for Gauss indices (g1, g2).
template <typename T>
__device__ __forceinline__ void moment4(T (&q)[4], int g1, int g2, T s) {
  q[0] += s;
  if (g1 != 1) q[1] = fma(gt<T>(g1), s, q[1]);
  if (g2 != 1) q[2] = fma(gt<T>(g2), s, q[2]);
  if (g1 != 1 && g2 != 1) q[3] = fma(T(gtd(g1) * gtd(g2)), s, q[3]);
}

// A[s1][s2] = (Q0/4 + s1 Q1/2 + s2 Q2/2 + s1 s2 Q3) / h, s = -1 (index 0) or +1 (index 1).
template <typename T>
__device__ __forceinline__ void inv_butterfly(const T (&Q)[4], T ih, T (&A)[2][2]) {
  const T q0 = Q[0] * (T(0.25) * ih), q1 = Q[1] * (T(0.5) * ih);
  const T q2 = Q[2] * (T(0.5) * ih), q3 = Q[3] * ih;
  const T r0m = q0 - q2, r0p = q0 + q2, r1m = q1 - q3, r1p = q1 + q3;
  A[0][0] = r0m - r1m;
  A[1][0] = r0m + r1m;
  A[0][1] = r0p - r1p;
  A[1][1] = r0p + r1p;
}

// (s0 a0 + s1 a1) + s2 a2 with s = -1 for index 0 and +1 for index 1, written with
// subtractions instead of negations (bit-identical: negation is exact and rounding
// is sign-symmetric).
template <typename T>
__device__ __forceinline__ T signed_sum3(T a0, T a1, T a2, int i, int j, int k) {
  if (i && j) return k ? (a0 + a1) + a2 : (a0 + a1) - a2;
  if (i) return k ? (a0 - a1) + a2 : (a0 - a1) - a2;
  if (j) return k ? (a1 - a0) + a2 : (a1 - a0) - a2;
  return k ? a2 - (a0 + a1) : -((a0 + a1) + a2);
}

// Modal sums: modal8 without the halvings, m'[p] = 2^(3 - popcount p) m[p] exactly
// (every intermediate is the mean form scaled by a power of two).
template <typename T>
__device__ __forceinline__ void modal8s(const T (&f)[8], T (&m)[8]) {
  T a[8], b[8];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    a[2 * p] = f[2 * p] + f[2 * p + 1];
    a[2 * p + 1] = f[2 * p + 1] - f[2 * p];
  }
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int al = 0; al < 2; al++) {
      T lo = a[al + 4 * k], hi = a[al + 2 + 4 * k];
      b[al + 4 * k] = lo + hi;
      b[al + 2 + 4 * k] = hi - lo;
    }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    T lo = b[q], hi = b[q + 4];
    m[q] = lo + hi;
    m[q + 4] = hi - lo;
  }
}

// a + b (2 t_g): the polynomials of the modal sums in the doubled coordinate 2t.
template <typename T> __device__ __forceinline__ T lin2(int g, T a, T b) {
  return g == 1 ? a : (g == 0 ? fma(b, T(-2 * VF_TAU), a) : fma(b, T(2 * VF_TAU), a));
}

// q[0..3] += s * {1, 2t1, 2t2, 4 t1 t2} for Gauss indices (g1, g2).
template <typename T>
__device__ __forceinline__ void moment4s(T (&q)[4], int g1, int g2, T s) {
  q[0] += s;
  if (g1 != 1) q[1] = fma(T(2 * gtd(g1)), s, q[1]);
  if (g2 != 1) q[2] = fma(T(2 * gtd(g2)), s, q[2]);
  if (g1 != 1 && g2 != 1) q[3] = fma(T(4 * gtd(g1) * gtd(g2)), s, q[3]);
}

// Node values of component c from the monomial coefficients w[p] (p = set of axes,
// w[0] unused) of the node polynomial in the signs (s_i, s_j, s_k) = +-1: a 3-stage
// signed butterfly.
template <typename T>
__device__ __forceinline__ void node_butterfly(const T (&w)[8], int c, T (&y)[8][3]) {
  // k: b[p][k] = w[p] -+ w[p + 4] (w[0] = 0)
  T b[4][2], d[2][2][2];
  b[0][0] = -w[4];
  b[0][1] = w[4];
#pragma unroll
  for (int p = 1; p < 4; p++) {
    b[p][0] = w[p] - w[p + 4];
    b[p][1] = w[p] + w[p + 4];
  }
  // j: d[p][j][k] = b[p][k] -+ b[p + 2][k]
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int p = 0; p < 2; p++) {
      d[p][0][k] = b[p][k] - b[p + 2][k];
      d[p][1][k] = b[p][k] + b[p + 2][k];
    }
  // i
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      y[2 * j + 4 * k][c] = d[0][j][k] - d[1][j][k];
      y[1 + 2 * j + 4 * k][c] = d[0][j][k] + d[1][j][k];
    }
}

// y[a][c] = (K_e(v) x_e)[a][c] for one element.
//
// Along a Gauss row (fixed gy, gz) the gradient is G(t) = G0 + t G1 in t = tx, with
// G1 having no x column, and v(t)^2 + eta = a0 + a1 t + a2 t^2, so the stress of
// every point is (a0 + a1 t + a2 t^2)(D0 + t D1), D = lambda tr(G) I + mu (G + G^T).
// The two sums over the row's three points that the moments need,
//   M0 = sum_gx w_x s = Wr [(a0 + a2/12) D0 + (a1/12) D1],
//   M1 = sum_gx w_x t s = Wr [(a1/12) D0 + ((a0 + 0.15 a2)/12) D1],
// follow from sum w_x = 1, sum w_x t^2 = 1/12, sum w_x t^4 = 1/80 (the odd sums
// vanish): the same 3-point Gauss sum as point by point, in about 2/3 of the
// operations.  Wr = vol w_y w_z.
//
// Scaling.  The element works on the modal sums (modal8s) in the doubled coordinate
// 2t, where the gradient column d is exactly G'/(4 h_d) and v is v'/8; the moments
// are taken against 2t as well (Q1' = 2 Q1, Q3' = 4 Q3), so the inverse butterfly
// needs no halvings either and node values are (Q0 +- Q1' +- Q2' +- Q3')/(4 h_d).
// With A0 = q0'^2 + 64 eta, A2 = q1'^2, H1 = q0' q1' (q0' + 2t q1' = 8 v along the
// row) the row scalars are C0 = W (A0 + A2/3), C1 = W 2 H1/3, E1 = W (A0 + 0.6 A2)/3
// with W = Wr/64, and M0, 2 M1 = C0 D0' + C1 D1', C1 D0' + E1 D1' (D1' = D(G1)/2).
// On cubic cells (CUBIC) every 1/(4h) factor is the same, so they all fold into W
// (W = Wr/(1024 h^2)); otherwise the gradient columns and the node values carry
// their own ih_d/4.  All the dropped halvings are powers of two: exact.
// VFGPU_U_GENERAL_NOINLINE (build option): the row closed form as a called function
// rather than inlined, so that a kernel capped at fewer registers than it needs spills
// only inside it (the fixed-weight element of the intact bulk stays spill-free).
#ifdef VFGPU_U_GENERAL_NOINLINE
#define VFGPU_U_GENERAL_INLINE __noinline__
#else
#define VFGPU_U_GENERAL_INLINE __forceinline__
#endif
template <typename T, bool CUBIC = false>
__device__ VFGPU_U_GENERAL_INLINE void u_element(const T (&xn)[8][3], const T (&vn)[8], T lam, T mu,
                                          T eta, T ihx, T ihy, T ihz, T vol, T (&y)[8][3]) {
  T m[3][8], mv[8];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    T f[8];
#pragma unroll
    for (int a = 0; a < 8; a++) f[a] = xn[a][c];
    modal8s(f, m[c]);
  }
  modal8s(vn, mv);
  // QX, QY, QZ: the 4 bilinear moments per component of the x, y, z stress columns.
  // SY0/SY1: M0/2M1 of the y column summed over the rows of a plane; SZ0/SZ1[c][gy]:
  // M0/2M1 of the z column summed over the planes, per row index.
  T QX[3][4], QY[3][4], QZ[3][4], SZ0[3][3], SZ1[3][3];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int q = 0; q < 4; q++) QX[c][q] = QY[c][q] = QZ[c][q] = T(0);
  const T mu2 = T(2) * mu, eta64 = T(64) * eta;
  const T sx = T(0.25) * ihx, sy = T(0.25) * ihy, sz = T(0.25) * ihz;
  const T wsc = CUBIC ? vol * (ihx * ihx) * T(1.0 / 1024.0) : vol * T(1.0 / 64.0);

#pragma unroll
  for (int gz = 0; gz < 3; gz++) {
    const T volw = wsc * gw<T>(gz);
    T ax[3], bx[3], ay[3], by[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T t37 = lin2(gz, m[c][3], m[c][7]);
      if (CUBIC) {
        ax[c] = lin2(gz, m[c][1], m[c][5]);
        bx[c] = t37;
        ay[c] = lin2(gz, m[c][2], m[c][6]);
        by[c] = t37;
      } else {
        ax[c] = lin2(gz, m[c][1], m[c][5]) * sx;
        bx[c] = t37 * sx;
        ay[c] = lin2(gz, m[c][2], m[c][6]) * sy;
        by[c] = t37 * sy;
      }
    }
    const T p0 = lin2(gz, mv[0], mv[4]), p1 = lin2(gz, mv[1], mv[5]);
    const T p2 = lin2(gz, mv[2], mv[6]), p3 = lin2(gz, mv[3], mv[7]);
    // D1' = D(G1') with G1' = [0 | by | be]: the y part is constant over the plane
    const T e01y = mu * by[0];
    T SY0[3], SY1[3];
#pragma unroll
    for (int gy = 0; gy < 3; gy++) {
      T Gx[3], al[3], be[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        Gx[c] = lin2(gy, ax[c], bx[c]);
        al[c] = lin2(gy, m[c][4], m[c][6]);
        be[c] = lin2(gy, m[c][5], m[c][7]);
        if (!CUBIC) {
          al[c] = al[c] * sz;
          be[c] = be[c] * sz;
        }
      }
      const T q0 = lin2(gy, p0, p2), q1 = lin2(gy, p1, p3);
      const T A0 = fma(q0, q0, eta64), A2 = q1 * q1, H1 = q0 * q1;
      const T C0 = (volw * T(gwd(gy))) * fma(A2, T(1.0 / 3.0), A0);
      const T C1 = (volw * T(gwd(gy) * (2.0 / 3.0))) * H1;
      const T E1 = (volw * T(gwd(gy) * (1.0 / 3.0))) * fma(A2, T(0.6), A0);
      // D0' = D(G0'), G0' = [Gx | ay | al]
      const T L0 = lam * ((Gx[0] + ay[1]) + al[2]);
      const T d00 = fma(mu2, Gx[0], L0), d11 = fma(mu2, ay[1], L0), d22 = fma(mu2, al[2], L0);
      const T d01 = mu * (ay[0] + Gx[1]), d02 = mu * (al[0] + Gx[2]), d12 = mu * (al[1] + ay[2]);
      // D1'
      const T L1 = lam * (by[1] + be[2]);
      const T e11 = fma(mu2, by[1], L1), e22 = fma(mu2, be[2], L1);
      const T e02 = mu * be[0], e12 = mu * (be[1] + by[2]);
      // M0 of the 6 stress components, 2 M1 of the 5 the y and z columns need
      const T n00 = fma(C0, d00, C1 * L1), n01 = fma(C0, d01, C1 * e01y);
      const T n02 = fma(C0, d02, C1 * e02), n11 = fma(C0, d11, C1 * e11);
      const T n12 = fma(C0, d12, C1 * e12), n22 = fma(C0, d22, C1 * e22);
      const T o01 = fma(C1, d01, E1 * e01y), o02 = fma(C1, d02, E1 * e02);
      const T o11 = fma(C1, d11, E1 * e11), o12 = fma(C1, d12, E1 * e12);
      const T o22 = fma(C1, d22, E1 * e22);
      moment4s(QX[0], gy, gz, n00);
      moment4s(QX[1], gy, gz, n01);
      moment4s(QX[2], gy, gz, n02);
      if (gy == 0) {
        SY0[0] = n01; SY0[1] = n11; SY0[2] = n12;
        SY1[0] = o01; SY1[1] = o11; SY1[2] = o12;
      } else {
        SY0[0] += n01; SY0[1] += n11; SY0[2] += n12;
        SY1[0] += o01; SY1[1] += o11; SY1[2] += o12;
      }
      if (gz == 0) {
        SZ0[0][gy] = n02; SZ0[1][gy] = n12; SZ0[2][gy] = n22;
        SZ1[0][gy] = o02; SZ1[1][gy] = o12; SZ1[2][gy] = o22;
      } else {
        SZ0[0][gy] += n02; SZ0[1][gy] += n12; SZ0[2][gy] += n22;
        SZ1[0][gy] += o02; SZ1[1][gy] += o12; SZ1[2][gy] += o22;
      }
    }
    // QY moments {1, 2tx, 2tz, 4 tx tz}: the 2tx moment is 2 M1
#pragma unroll
    for (int c = 0; c < 3; c++) {
      QY[c][0] += SY0[c];
      QY[c][1] += SY1[c];
      if (gz != 1) {
        QY[c][2] = fma(T(2 * gtd(gz)), SY0[c], QY[c][2]);
        QY[c][3] = fma(T(2 * gtd(gz)), SY1[c], QY[c][3]);
      }
    }
  }
  // QZ moments {1, 2tx, 2ty, 4 tx ty}
#pragma unroll
  for (int gy = 0; gy < 3; gy++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      QZ[c][0] += SZ0[c][gy];
      QZ[c][1] += SZ1[c][gy];
      if (gy != 1) {
        QZ[c][2] = fma(T(2 * gtd(gy)), SZ0[c][gy], QZ[c][2]);
        QZ[c][3] = fma(T(2 * gtd(gy)), SZ1[c][gy], QZ[c][3]);
      }
    }

  // Back to the nodes.  The direction-d part of node (i,j,k) is
  //   s_d (Q0 + s_1 Q1' + s_2 Q2' + s_1 s_2 Q3') / (4 h_d), s = -1 (node 0) or +1 (node 1),
  // so y_ijk is a polynomial in (s_i, s_j, s_k) with the monomial coefficients
  //   s_i: QX0, s_j: QY0, s_k: QZ0, s_i s_j: QX1 + QY1, s_i s_k: QX2 + QZ1,
  //   s_j s_k: QY2 + QZ2, s_i s_j s_k: QX3 + QY3 + QZ3 (each Q times its ih_d/4),
  // evaluated at the 8 sign patterns by a 3-stage signed butterfly.
#pragma unroll
  for (int c = 0; c < 3; c++) {
    T w[8];
    if (CUBIC) {
      w[1] = QX[c][0];
      w[2] = QY[c][0];
      w[3] = QX[c][1] + QY[c][1];
      w[4] = QZ[c][0];
      w[5] = QX[c][2] + QZ[c][1];
      w[6] = QY[c][2] + QZ[c][2];
      w[7] = (QX[c][3] + QY[c][3]) + QZ[c][3];
    } else {
      w[1] = QX[c][0] * sx;
      w[2] = QY[c][0] * sy;
      w[3] = fma(QX[c][1], sx, QY[c][1] * sy);
      w[4] = QZ[c][0] * sz;
      w[5] = fma(QX[c][2], sx, QZ[c][1] * sz);
      w[6] = fma(QY[c][2], sy, QZ[c][2] * sz);
      w[7] = fma(QX[c][3], sx, fma(QY[c][3], sy, QZ[c][3] * sz));
    }
    node_butterfly(w, c, y);
  }
}

// Element with a constant phase field.
//
// Where the 8 nodal v of an element are equal, v^2 + eta = S at every point and the
// stress S D(G) is a polynomial of degree <= 1 per axis in each column, so its moments
// against {1, s_a, s_b, s_a s_b} (doubled coordinate s = 2t) are exact cell averages:
// E[s^2] = 1/3 and odd moments vanish -- what the reference's 3-point Gauss sum gives
// for these degrees, without evaluating any point.  With the modal sums m (modal8s),
// k_d = 1/(4 h_d) and the gradient coefficients G[c][d][B] = m[c][B + d] k_d of the
// monomial s^B (B a set of axes without d):
//   T_B = sum_{e not in B} G[e][e][B]                 (trace coefficient of s^B)
//   R[c][d][B] = vol S 3^-|B| k_d [lambda [c == d] T_B
//                + mu (G[c][d][B] + [c not in B] G[d][c][B])],
// and the node polynomial of component c has the coefficient w[p] = sum_{d in p}
// R[c][d][p - d] for the monomial p (the same signed butterfly as u_element).  On cubic
// cells every k folds into the weight.  About 240 operations per element against ~925 for
// u_element; equal to it up to rounding.
// A product the compiler may not contract into a later add (f2's overload is in f2.cuh).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <typename T, bool CUBIC = false>
__device__ __forceinline__ void u_element_const(const T (&xn)[8][3], T S, T lam, T mu, T ihx,
                                                T ihy, T ihz, T vol, T (&y)[8][3]) {
  T m[3][8];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    T f[8];
#pragma unroll
    for (int a = 0; a < 8; a++) f[a] = xn[a][c];
    modal8s(f, m[c]);
  }
  const T k[3] = {T(0.25) * ihx, T(0.25) * ihy, T(0.25) * ihz};
  // gradient coefficient of component c, direction d, monomial B (as m * k unless CUBIC)
  auto gm = [&](int c, int d, int B) -> T { return m[c][B | (1 << d)]; };
  auto G = [&](int c, int d, int B) -> T { return CUBIC ? gm(c, d, B) : gm(c, d, B) * k[d]; };
  // Every multiply that feeds an add is an explicit fma, or a product the compiler may
  // not fuse (mul_rn: it reaches the adds below and the node butterfly's), so nothing is
  // left to contract: the scalar and the packed two-lane (f2) builds of this element give
  // the same bits per lane.
  T tr[7];
#pragma unroll
  for (int B = 0; B < 7; B++) {
    T t = T(0);
    bool first = true;
#pragma unroll
    for (int e = 0; e < 3; e++)
      if (!((B >> e) & 1)) {
        if (CUBIC) t = first ? gm(e, e, B) : t + gm(e, e, B);
        else t = first ? gm(e, e, B) * k[e] : fma(gm(e, e, B), k[e], t);
        first = false;
      }
    tr[B] = t;
  }
  const T W0 = CUBIC ? (vol * S) * (k[0] * k[0]) : vol * S;
  const T Wn[3] = {W0, W0 * T(1.0 / 3.0), W0 * T(1.0 / 9.0)};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    T w[8];
    w[0] = T(0);
#pragma unroll
    for (int p = 1; p < 8; p++) {
      T acc = T(0);
      bool first = true;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (!((p >> d) & 1)) continue;
        const int B = p & ~(1 << d);
        const int nb = (B & 1) + ((B >> 1) & 1) + ((B >> 2) & 1);
        const T Wd = CUBIC ? Wn[nb] : Wn[nb] * k[d];
        if (c == d) {
          const T R = fma(T(2) * mu * Wd, G(c, c, B), (lam * Wd) * tr[B]);
          acc = first ? R : acc + R;
        } else {
          T g;  // the symmetric gradient pair, or the one coefficient present
          if (!((B >> c) & 1))
            g = CUBIC ? gm(c, d, B) + gm(d, c, B) : fma(gm(d, c, B), k[c], gm(c, d, B) * k[d]);
          else
            g = G(c, d, B);
          const T s = mu * Wd;
          acc = first ? mul_rn(s, g) : fma(s, g, acc);
        }
        first = false;
      }
      w[p] = acc;
    }
    node_butterfly(w, c, y);
  }
}

// The NOCOMPRESSION operator K(v; u0) (VF_BilinearFormUNoCompression3D_local,
// VFMech.c:299-376) for one element: at Gauss point g, if bit g of `flags` is set
// (tr(eps(u0)) < 0 there) the spherical part keeps kappa (1 + eta), so the stress is
//   w [lambda' tr(G) I + s mu (G + G^T)],  lambda' = kappa (1 + eta) - 2 mu s / 3,
// and otherwise the plain w s (lambda tr(G) I + mu (G + G^T)).  The coefficient is
// no longer one polynomial along a row, so this variant sums point by point (same
// modal gradients and moments as u_element); the z moments are accumulated at every
// point to keep the register count down.
template <typename T>
__device__ __forceinline__ void u_element_nc(const T (&xn)[8][3], const T (&vn)[8], T lam, T mu,
                                             T eta, T ihx, T ihy, T ihz, T vol, uint32_t flags,
                                             T (&y)[8][3]) {
  T m[3][8], mv[8];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    T f[8];
#pragma unroll
    for (int a = 0; a < 8; a++) f[a] = xn[a][c];
    modal8(f, m[c]);
  }
  modal8(vn, mv);
  T QX[3][4], QY[3][4], QZ[3][4];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int q = 0; q < 4; q++) QX[c][q] = QY[c][q] = QZ[c][q] = T(0);
  const T mu2 = T(2) * mu, kap1 = (lam + T(2.0 / 3.0) * mu) * (T(1) + eta), mu23 = T(2.0 / 3.0) * mu;
#pragma unroll
  for (int gz = 0; gz < 3; gz++) {
    const T volw = vol * gw<T>(gz);
    T ax[3], bx[3], ay[3], by[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T t37 = lin(gz, m[c][3], m[c][7]);
      ax[c] = lin(gz, m[c][1], m[c][5]) * ihx;
      bx[c] = t37 * ihx;
      ay[c] = lin(gz, m[c][2], m[c][6]) * ihy;
      by[c] = t37 * ihy;
    }
    const T p0 = lin(gz, mv[0], mv[4]), p1 = lin(gz, mv[1], mv[5]);
    const T p2 = lin(gz, mv[2], mv[6]), p3 = lin(gz, mv[3], mv[7]);
    T SY[3][3];
#pragma unroll
    for (int gy = 0; gy < 3; gy++) {
      T Gx[3], al[3], be[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        Gx[c] = lin(gy, ax[c], bx[c]);
        al[c] = lin(gy, m[c][4], m[c][6]) * ihz;
        be[c] = lin(gy, m[c][5], m[c][7]) * ihz;
      }
      const T q0 = lin(gy, p0, p2), q1 = lin(gy, p1, p3);
      T SX[3];
#pragma unroll
      for (int gx = 0; gx < 3; gx++) {
        T Gy[3], Gz[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          Gy[c] = lin(gx, ay[c], by[c]);
          Gz[c] = lin(gx, al[c], be[c]);
        }
        const T vg = lin(gx, q0, q1);
        const T sv = fma(vg, vg, eta);
        const T wq = volw * T(gwd(gx) * gwd(gy));
        const T ws = wq * sv;
        const T tr = Gx[0] + Gy[1] + Gz[2];
        const bool comp = (flags >> (gx + 3 * gy + 9 * gz)) & 1u;
        const T L = comp ? (wq * (kap1 - mu23 * sv)) * tr : (ws * lam) * tr;
        const T m2 = ws * mu2, m1 = ws * mu;
        const T s00 = fma(m2, Gx[0], L), s11 = fma(m2, Gy[1], L), s22 = fma(m2, Gz[2], L);
        const T s01 = m1 * (Gy[0] + Gx[1]);
        const T s02 = m1 * (Gz[0] + Gx[2]);
        const T s12 = m1 * (Gz[1] + Gy[2]);
        if (gx == 0) {
          SX[0] = s00; SX[1] = s01; SX[2] = s02;
        } else {
          SX[0] += s00; SX[1] += s01; SX[2] += s02;
        }
        if (gy == 0) {
          SY[0][gx] = s01; SY[1][gx] = s11; SY[2][gx] = s12;
        } else {
          SY[0][gx] += s01; SY[1][gx] += s11; SY[2][gx] += s12;
        }
        moment4(QZ[0], gx, gy, s02);
        moment4(QZ[1], gx, gy, s12);
        moment4(QZ[2], gx, gy, s22);
      }
#pragma unroll
      for (int c = 0; c < 3; c++) moment4(QX[c], gy, gz, SX[c]);
    }
#pragma unroll
    for (int gx = 0; gx < 3; gx++)
#pragma unroll
      for (int c = 0; c < 3; c++) moment4(QY[c], gx, gz, SY[c][gx]);
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    T A[3][2][2];
    inv_butterfly(QX[c], ihx, A[0]);
    inv_butterfly(QY[c], ihy, A[1]);
    inv_butterfly(QZ[c], ihz, A[2]);
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
      for (int j = 0; j < 2; j++)
#pragma unroll
        for (int i = 0; i < 2; i++)
          y[i + 2 * j + 4 * k][c] = signed_sum3(A[0][j][k], A[1][i][k], A[2][i][j], i, j, k);
  }
}

}  // namespace vfgpu
