// ops.cuh -- element operators plugged into the tile engine.
//
//   UOp: y = K(v) x, the degraded elasticity operator of VF_BilinearFormU3D_local
//        (VFMech.c:227-290) with Dirichlet rows identity (VFCartFE.c:1147-1296).
//   VOp: y = K_V x, the damage operator of VF_BilinearFormVAT1/AT23D_local +
//        VF_BilinearFormVCoupling3D_local (VFMech.c:2040-2115):
//        (Gc/(2 c_w)) eps int grad(phi_a).grad(phi_b) + int c(x) phi_a phi_b,
//        c = 2 W(u) [+ Gc/(2 c_w)/eps for AT2], with c premultiplied by the Gauss
//        weight and stored per element and Gauss point (vfgpu v_coef kernel); the
//        tile engine stages each element layer's 27 values per cell into shared
//        memory with one 3-D tensor copy (cmap), two layers ahead of use.
//        An optional mask removes dofs (row and column) for the reduced-space
//        solves of the VI Newton method and the rows+columns Dirichlet/irreversibility
//        treatment (VFCartFE.c:1305-1454, VFMech.c:2637-2682).
#pragma once

#include "f2.cuh"
#include "tile_engine.cuh"
#include "u_apply.cuh"

// Build option: the fixed-weight U wave copies its node planes with 1-D tensor copies, two
// per tile row (PlaneBox), instead of one cp.async per value.  Bit-identical; measured
// slower on B200 at 129^3 on the penny field (FP64 apply 0.1223 ms against 0.1167, FP32
// 0.0872 against 0.0855; with one thread waiting on each plane's mbarrier 0.1236 ms).
#ifndef VFGPU_U_PLANES_TMA
#define VFGPU_U_PLANES_TMA 0
#endif

namespace vfgpu {

// CUBIC: hx = hy = hz, every 1/h factor folds into the row weight (u_element).
template <typename T_, bool CUBIC = false> struct UOp {
  using T = T_;
  using Args = UApplyArgs<T>;
  static constexpr int NC = 3, NIN = 4, EPT = 1, CV = 0;
  static constexpr int LIST = 1;  // the unit list this operator takes in a split launch
  static constexpr bool PLANES_TMA = false;  // node planes by cp.async values
  __device__ __forceinline__ static void node_src(const Args& A, int64_t n, const T* (&src)[NIN]) {
    src[0] = A.x + 3 * n;
    src[1] = A.x + 3 * n + 1;
    src[2] = A.x + 3 * n + 2;
    src[3] = A.v + n;
  }
  // The cell's Lame coefficients (material layer table, or per-cell modulus).
  __device__ __forceinline__ static void lame(const Args& A, const LayerTable& L, int ex, int ey,
                                              int ez, T& lam, T& mu) {
    const int layer = A.elayer ? A.elayer[ez] : 0;
    const LayerTable& LT = A.P ? A.P->L : L;
    if (A.cellE) {
      const T E = T(A.cellE[((int64_t)ez * (A.ny - 1) + ey) * (A.nx - 1) + ex]);
      lam = E * T(LT.lamfac[layer]);
      mu = E * T(LT.mufac[layer]);
    } else {
      lam = T(LT.lambda[layer]);
      mu = T(LT.mu[layer]);
    }
  }
  __device__ __forceinline__ static T eta_of(const Args& A) { return A.P ? T(A.P->eta) : A.eta; }
  __device__ __forceinline__ static void element(const Args& A, const LayerTable& L, int ex,
                                                 int ey, int ez, const T (&in)[8][NIN],
                                                 T (&out)[8][NC]) {
    T xn[8][3], vn[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
      xn[a][0] = in[a][0];
      xn[a][1] = in[a][1];
      xn[a][2] = in[a][2];
      vn[a] = in[a][3];
    }
    T lam, mu;
    lame(A, L, ex, ey, ez, lam, mu);
    const T eta = eta_of(A);
    // an element whose nodal phase field is constant (the intact bulk, v = 1) takes the
    // fixed-weight form; the rest the row closed form
    const T v0 = vn[0];
    bool cst = true;
#pragma unroll
    for (int a = 1; a < 8; a++) cst = cst && vn[a] == v0;
    if (cst)
      u_element_const<T, CUBIC>(xn, fma(v0, v0, eta), lam, mu, A.ihx, A.ihy, A.ihz, A.vol, out);
    else
      u_element<T, CUBIC>(xn, vn, lam, mu, eta, A.ihx, A.ihy, A.ihz, A.vol, out);
  }
  // The same for an element known to have a constant nodal phase field (the choice
  // element makes for it, without the general form in the code path).
  __device__ __forceinline__ static void element_const(const Args& A, const LayerTable& L, int ex,
                                                       int ey, int ez, const T (&in)[8][NIN],
                                                       T (&out)[8][NC]) {
    T xn[8][3];
#pragma unroll
    for (int a = 0; a < 8; a++) {
      xn[a][0] = in[a][0];
      xn[a][1] = in[a][1];
      xn[a][2] = in[a][2];
    }
    T lam, mu;
    lame(A, L, ex, ey, ez, lam, mu);
    const T v0 = in[0][3];
    u_element_const<T, CUBIC>(xn, fma(v0, v0, eta_of(A)), lam, mu, A.ihx, A.ihy, A.ihz, A.vol, out);
  }
  // The per-node flags finish_node needs (Dirichlet bits), loaded ahead by the tiles.
  __device__ __forceinline__ static unsigned node_flags(const Args& A, int64_t n) {
    return A.bc ? A.bc[n] : 0u;
  }
  // Writes y of node n (Dirichlet rows: y = x) from the node's flags b and input
  // values xin; with DOT, returns x.y over its dofs (the launch accumulates the CG dot
  // into A.dot).
  template <bool DOT>
  __device__ __forceinline__ static double finish_node_in(const Args& A, int64_t n, const T (&val)[NC],
                                                          unsigned b, const T (&xin)[NC]) {
    double d = 0.;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T y = ((b >> c) & 1u) ? xin[c] : val[c];
      A.y[3 * n + c] = y;
      if constexpr (DOT) d += (double)xin[c] * (double)y;
    }
    return d;
  }
  // The same with the flags and inputs read from global memory (the seam fix-up).
  template <bool DOT>
  __device__ __forceinline__ static double finish_node(const Args& A, int64_t n, const T (&val)[NC]) {
    const unsigned b = node_flags(A, n);
    T xin[NC];
#pragma unroll
    for (int c = 0; c < 3; c++) xin[c] = (DOT || ((b >> c) & 1u)) ? A.x[3 * n + c] : T(0);
    return finish_node_in<DOT>(A, n, val, b, xin);
  }
};

// UOp for the units of unit list 0, whose elements all have a constant nodal phase
// field: the fixed-weight element alone (the choice UOp::element makes for them, with
// the same arithmetic), compiled without the general element.
template <typename T_, bool CUBIC = false> struct UOpConst : UOp<T_, CUBIC> {
  using Base = UOp<T_, CUBIC>;
  using T = T_;
  using Args = UApplyArgs<T>;
  static constexpr int LIST = 0;
  static constexpr bool PLANES_TMA = VFGPU_U_PLANES_TMA != 0;  // node planes by tensor copies
  __device__ __forceinline__ static void element(const Args& A, const LayerTable& L, int ex,
                                                 int ey, int ez, const T (&in)[8][Base::NIN],
                                                 T (&out)[8][Base::NC]) {
    Base::element_const(A, L, ex, ey, ez, in, out);
  }
};

// The NOCOMPRESSION U operator: UOp with the per-point element u_element_nc and the
// per-cell compression bits A.cflag.
template <typename T_> struct UOpNC {
  using T = T_;
  using Args = UApplyArgs<T>;
  static constexpr int NC = 3, NIN = 4, EPT = 1, CV = 0;
  static constexpr int LIST = -1;
  static constexpr bool PLANES_TMA = false;
  __device__ __forceinline__ static void node_src(const Args& A, int64_t n, const T* (&src)[NIN]) {
    UOp<T>::node_src(A, n, src);
  }
  __device__ __forceinline__ static void element(const Args& A, const LayerTable& L, int ex,
                                                 int ey, int ez, const T (&in)[8][NIN],
                                                 T (&out)[8][NC]) {
    T xn[8][3], vn[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
      xn[a][0] = in[a][0];
      xn[a][1] = in[a][1];
      xn[a][2] = in[a][2];
      vn[a] = in[a][3];
    }
    const int layer = A.elayer ? A.elayer[ez] : 0;
    const LayerTable& LT = A.P ? A.P->L : L;
    const T eta = A.P ? T(A.P->eta) : A.eta;
    const int64_t cell = ((int64_t)ez * (A.ny - 1) + ey) * (A.nx - 1) + ex;
    T lam, mu;
    if (A.cellE) {
      const T E = T(A.cellE[cell]);
      lam = E * T(LT.lamfac[layer]);
      mu = E * T(LT.mufac[layer]);
    } else {
      lam = T(LT.lambda[layer]);
      mu = T(LT.mu[layer]);
    }
    u_element_nc<T>(xn, vn, lam, mu, eta, A.ihx, A.ihy, A.ihz, A.vol, A.cflag[cell], out);
  }
  __device__ __forceinline__ static unsigned node_flags(const Args& A, int64_t n) {
    return UOp<T>::node_flags(A, n);
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node_in(const Args& A, int64_t n, const T (&val)[NC],
                                                          unsigned b, const T (&xin)[NC]) {
    return UOp<T>::template finish_node_in<DOT>(A, n, val, b, xin);
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node(const Args& A, int64_t n, const T (&val)[NC]) {
    return UOp<T>::template finish_node<DOT>(A, n, val);
  }
};

// The FP32 U operator on two y-adjacent elements per thread, one per lane of the
// packed FP32 instructions (f2): the same arithmetic as UOp<float> with half the
// instructions.
struct UOpF2 {
  using T = float;
  using Args = UApplyArgs<float>;
  static constexpr int NC = 3, NIN = 4, EPT = 2, CV = 0;
  static constexpr int LIST = -1;
  static constexpr bool PLANES_TMA = false;
  __device__ __forceinline__ static void node_src(const Args& A, int64_t n, const T* (&src)[NIN]) {
    UOp<float>::node_src(A, n, src);
  }
  __device__ __forceinline__ static void element_multi(const Args& A, const LayerTable& L, int ex,
                                                       const int (&ey)[2], int ez, const bool (&ok)[2],
                                                       const T (&in)[2][8][NIN], T (&out)[2][8][NC]) {
    f2 xn[8][3], vn[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
#pragma unroll
      for (int c = 0; c < 3; c++) xn[a][c] = f2(in[0][a][c], in[1][a][c]);
      vn[a] = f2(in[0][a][3], in[1][a][3]);
    }
    const int layer = A.elayer ? A.elayer[ez] : 0;
    const LayerTable& LT = A.P ? A.P->L : L;
    const float eta = A.P ? float(A.P->eta) : A.eta;
    f2 lam, mu;
    if (A.cellE) {
      float E[2];
#pragma unroll
      for (int e = 0; e < 2; e++)
        E[e] = ok[e] ? A.cellE[((int64_t)ez * (A.ny - 1) + ey[e]) * (A.nx - 1) + ex] : 0.f;
      const f2 Ep(E[0], E[1]);
      lam = Ep * f2(float(LT.lamfac[layer]));
      mu = Ep * f2(float(LT.mufac[layer]));
    } else {
      lam = f2(float(LT.lambda[layer]));
      mu = f2(float(LT.mu[layer]));
    }
    f2 y[8][3];
    u_element<f2>(xn, vn, lam, mu, f2(eta), f2(A.ihx), f2(A.ihy), f2(A.ihz), f2(A.vol), y);
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        out[0][a][c] = ok[0] ? y[a][c].v.x : 0.f;
        out[1][a][c] = ok[1] ? y[a][c].v.y : 0.f;
      }
  }
  __device__ __forceinline__ static unsigned node_flags(const Args& A, int64_t n) {
    return UOp<float>::node_flags(A, n);
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node_in(const Args& A, int64_t n, const T (&val)[NC],
                                                          unsigned b, const T (&xin)[NC]) {
    return UOp<float>::finish_node_in<DOT>(A, n, val, b, xin);
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node(const Args& A, int64_t n, const T (&val)[NC]) {
    return UOp<float>::finish_node<DOT>(A, n, val);
  }
};

// UOpConst<float, CUBIC> on two y-adjacent elements per thread, one per lane of the
// packed FP32 instructions (f2): unit list 0 of the FP32 split.  u_element_const has no
// contractible multiply-add, so each lane gives the scalar kernel's bits.
template <bool CUBIC = false> struct UOpF2Const {
  using T = float;
  using Args = UApplyArgs<float>;
  static constexpr int NC = 3, NIN = 4, EPT = 2, CV = 0;
  static constexpr int LIST = 0;
  static constexpr bool PLANES_TMA = VFGPU_U_PLANES_TMA != 0;
  __device__ __forceinline__ static void node_src(const Args& A, int64_t n, const T* (&src)[NIN]) {
    UOp<float>::node_src(A, n, src);
  }
  __device__ __forceinline__ static void element_multi(const Args& A, const LayerTable& L, int ex,
                                                       const int (&ey)[2], int ez, const bool (&ok)[2],
                                                       const T (&in)[2][8][NIN], T (&out)[2][8][NC]) {
    f2 xn[8][3];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int c = 0; c < 3; c++) xn[a][c] = f2(in[0][a][c], in[1][a][c]);
    const int layer = A.elayer ? A.elayer[ez] : 0;
    const LayerTable& LT = A.P ? A.P->L : L;
    const float eta = A.P ? float(A.P->eta) : A.eta;
    f2 lam, mu;
    if (A.cellE) {
      float E[2];
#pragma unroll
      for (int e = 0; e < 2; e++)
        E[e] = ok[e] ? A.cellE[((int64_t)ez * (A.ny - 1) + ey[e]) * (A.nx - 1) + ex] : 0.f;
      const f2 Ep(E[0], E[1]);
      lam = Ep * f2(float(LT.lamfac[layer]));
      mu = Ep * f2(float(LT.mufac[layer]));
    } else {
      lam = f2(float(LT.lambda[layer]));
      mu = f2(float(LT.mu[layer]));
    }
    const f2 v0(in[0][0][3], in[1][0][3]);
    f2 y[8][3];
    u_element_const<f2, CUBIC>(xn, fma(v0, v0, f2(eta)), lam, mu, f2(A.ihx), f2(A.ihy), f2(A.ihz),
                               f2(A.vol), y);
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        out[0][a][c] = ok[0] ? y[a][c].v.x : 0.f;
        out[1][a][c] = ok[1] ? y[a][c].v.y : 0.f;
      }
  }
  __device__ __forceinline__ static unsigned node_flags(const Args& A, int64_t n) {
    return UOp<float>::node_flags(A, n);
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node_in(const Args& A, int64_t n, const T (&val)[NC],
                                                          unsigned b, const T (&xin)[NC]) {
    return UOp<float>::template finish_node_in<DOT>(A, n, val, b, xin);
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node(const Args& A, int64_t n, const T (&val)[NC]) {
    return UOp<float>::template finish_node<DOT>(A, n, val);
  }
};

template <typename T> struct VApplyArgs {
  CUtensorMap cmap;                   // the coefficient as a 3-D tensor (ex, ey, 27 ez + g),
                                      // box 32 x TY x 27 (vcoef_index layout)
  unsigned* __restrict__ cerr;        // set to 1 when a coefficient copy was not seen in time
  const T* __restrict__ x;            // N input; must be 0 on masked dofs (the reduced-space
                                      // CG keeps its directions 0 there), which makes the
                                      // masked columns drop out
  T* __restrict__ y;                  // N output
  const uint8_t* __restrict__ mask;   // N: nonzero => dof removed (y = 0); or null
  const uint8_t* __restrict__ elayer; // nz-1 or null
  T* __restrict__ seamX;
  T* __restrict__ seamY;
  const int* __restrict__ skip;       // if non-null and *skip != 0 the launch does nothing
  const DevParams* __restrict__ P;    // Gc/(2 c_w) eps per layer
  double* __restrict__ dot;           // if non-null: per-block partials of x.y
  int nx, ny, nz, ntx, nty;
  T ihx, ihy, ihz, vol;
};

// A[s1][s2] = q0 + s1 q1 + s2 q2 + s1 s2 q3, s = -1 (index 0) or +1 (index 1).
template <typename T>
__device__ __forceinline__ void butterfly4(T q0, T q1, T q2, T q3, T (&A)[2][2]) {
  const T r0m = q0 - q2, r0p = q0 + q2, r1m = q1 - q3, r1p = q1 + q3;
  A[0][0] = r0m - r1m;
  A[1][0] = r0m + r1m;
  A[0][1] = r0p - r1p;
  A[1][1] = r0p + r1p;
}

// y[a] = (K_V,e x_e)[a] for one element, in the modal form x = sum_p m_p t^p on the
// unit cell t in [-1/2, 1/2]^3 (modal8, as u_element):
//  - stiffness aeps int grad(phi_a).grad(x): the x-derivative is ihx (m1 + m3 ty +
//    m5 tz + m7 ty tz), and its moments against {1, ty, tz, ty tz} are exactly
//    {m1, m3 / 12, m5 / 12, m7 / 144} ihx (<t> = 0, <t^2> = 1/12), which is what the
//    reference's 27-point Gauss sum gives for this integrand (VF_BilinearFormVAT1/
//    AT23D_local, VFMech.c:2040-2115; 3 points per axis are exact for it), so the
//    closed form replaces the sum; likewise y and z;
//  - mass int c phi_a x with c given per Gauss point: x at the 27 points by sum
//    factorisation of the modal form, psi_g = c_g x_g, and the moments
//    M_p = sum_g psi_g t^p by sum factorisation along x, then y, then z.
template <typename T>
__device__ __forceinline__ void v_element(const T (&xn)[8], const T* __restrict__ cg, int cs,
                                          T aeps, T ihx, T ihy, T ihz, T vol, T (&y)[8]) {
  T m[8];
  modal8(xn, m);
  const T av = aeps * vol;
  const T kx = av * ihx * ihx, ky = av * ihy * ihy, kz = av * ihz * ihz;
  const T c4 = T(0.25), c24 = T(1.0 / 24.0), c144 = T(1.0 / 144.0);
  T AX[2][2], AY[2][2], AZ[2][2];
  butterfly4((kx * c4) * m[1], (kx * c24) * m[3], (kx * c24) * m[5], (kx * c144) * m[7], AX);
  butterfly4((ky * c4) * m[2], (ky * c24) * m[3], (ky * c24) * m[6], (ky * c144) * m[7], AY);
  butterfly4((kz * c4) * m[4], (kz * c24) * m[5], (kz * c24) * m[6], (kz * c144) * m[7], AZ);
  // per gz: sums over the (gx, gy) points of psi {1, ty, tx, tx ty}, each t as its sign
  T P00[3], P01[3], P10[3], P11[3];
#pragma unroll
  for (int gz = 0; gz < 3; gz++) {
    const T p0 = lin(gz, m[0], m[4]), p1 = lin(gz, m[1], m[5]);
    const T p2 = lin(gz, m[2], m[6]), p3 = lin(gz, m[3], m[7]);
    T L0[3], L1[3];
#pragma unroll
    for (int gy = 0; gy < 3; gy++) {
      const T q0 = lin(gy, p0, p2), q1 = lin(gy, p1, p3);
      T psi[3];
#pragma unroll
      for (int gx = 0; gx < 3; gx++) psi[gx] = cg[(gx + 3 * gy + 9 * gz) * cs] * lin(gx, q0, q1);
      L0[gy] = (psi[0] + psi[1]) + psi[2];
      L1[gy] = psi[2] - psi[0];
    }
    P00[gz] = (L0[0] + L0[1]) + L0[2];
    P01[gz] = L0[2] - L0[0];
    P10[gz] = (L1[0] + L1[1]) + L1[2];
    P11[gz] = L1[2] - L1[0];
  }
  const T t1 = T(VF_TAU), t2 = T(VF_TAU * VF_TAU), t3 = T(VF_TAU * VF_TAU * VF_TAU);
  T M[8];  // value moments sum psi P_a(tx) P_b(ty) P_c(tz)
  M[0] = (P00[0] + P00[1]) + P00[2];
  M[1] = t1 * ((P10[0] + P10[1]) + P10[2]);
  M[2] = t1 * ((P01[0] + P01[1]) + P01[2]);
  M[3] = t2 * ((P11[0] + P11[1]) + P11[2]);
  M[4] = t1 * (P00[2] - P00[0]);
  M[5] = t2 * (P10[2] - P10[0]);
  M[6] = t2 * (P01[2] - P01[0]);
  M[7] = t3 * (P11[2] - P11[0]);
  // value part: sum_g psi prod_d (1/2 + s_d t_d) -> 3 inverse butterflies over M
  T b1[8], b2[8], b3[8];
#pragma unroll
  for (int q = 0; q < 4; q++) {  // z: M[q] (mode 0), M[q+4] (mode 1) -> k = 0,1
    b1[q] = T(0.5) * M[q] - M[q + 4];
    b1[q + 4] = T(0.5) * M[q] + M[q + 4];
  }
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int al = 0; al < 2; al++) {  // y
      const T lo = b1[al + 4 * k], hi = b1[al + 2 + 4 * k];
      b2[al + 4 * k] = T(0.5) * lo - hi;
      b2[al + 2 + 4 * k] = T(0.5) * lo + hi;
    }
#pragma unroll
  for (int p = 0; p < 4; p++) {  // x
    const T lo = b2[2 * p], hi = b2[2 * p + 1];
    b3[2 * p] = T(0.5) * lo - hi;
    b3[2 * p + 1] = T(0.5) * lo + hi;
  }
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const T ax_ = i ? AX[j][k] : -AX[j][k];
        const T ay_ = j ? AY[i][k] : -AY[i][k];
        const T az_ = k ? AZ[i][j] : -AZ[i][j];
        y[i + 2 * j + 4 * k] = ((ax_ + ay_) + az_) + b3[i + 2 * j + 4 * k];
      }
}

template <typename T_> struct VOp {
  using T = T_;
  using Args = VApplyArgs<T>;
  static constexpr int NC = 1, NIN = 1, EPT = 1;
  static constexpr int LIST = -1;
  static constexpr bool PLANES_TMA = false;
  static constexpr int CV = 27;  // per-cell values staged by the engine (the coefficient)
  __device__ __forceinline__ static const CUtensorMap* cell_map(const Args& A) { return &A.cmap; }
  __device__ __forceinline__ static unsigned* cell_err(const Args& A) { return A.cerr; }
  __device__ __forceinline__ static void node_src(const Args& A, int64_t n, const T* (&src)[NIN]) {
    src[0] = A.x + n;
  }
  // cc: the element's 27 coefficients in shared memory, cs apart
  __device__ __forceinline__ static void element(const Args& A, const LayerTable& L, int ex,
                                                 int ey, int ez, const T (&in)[8][NIN],
                                                 T (&out)[8][NC], const T* cc, int cs) {
    T xn[8], yn[8];
#pragma unroll
    for (int a = 0; a < 8; a++) xn[a] = in[a][0];
    const int layer = A.elayer ? A.elayer[ez] : 0;
    v_element<T>(xn, cc, cs, T(A.P->aeps[layer]), A.ihx, A.ihy, A.ihz, A.vol, yn);
#pragma unroll
    for (int a = 0; a < 8; a++) out[a][0] = yn[a];
  }
  __device__ __forceinline__ static unsigned node_flags(const Args& A, int64_t n) {
    return A.mask ? A.mask[n] : 0u;
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node_in(const Args& A, int64_t n, const T (&val)[NC],
                                                          unsigned m, const T (&xin)[NC]) {
    const T y = m ? T(0) : val[0];
    A.y[n] = y;
    if constexpr (DOT) return (double)xin[0] * (double)y;
    return 0.;
  }
  template <bool DOT>
  __device__ __forceinline__ static double finish_node(const Args& A, int64_t n, const T (&val)[NC]) {
    const T xin[NC] = {DOT ? A.x[n] : T(0)};
    return finish_node_in<DOT>(A, n, val, node_flags(A, n), xin);
  }
};

}  // namespace vfgpu
