// elem.h -- once-per-solve element kernels (FP64): load vectors, Jacobi diagonals,
// the V coupling coefficient, energies and crack opening.
#pragma once

#include "common.cuh"

namespace vfgpu {

// VFCartFEElement3DInit tables (VFCartFE.c:216-269) of the uniform element.
struct ETab {
  double w[27];
  double phi[8][27];
  double dphi[8][3][27];
};
void etab_host(double hx, double hy, double hz, ETab* e);

struct ElemArgs {
  ETab tab;  // by value: the kernels read the tables from the parameter (constant) bank
  int nx, ny, nz;
  const uint8_t* __restrict__ elayer;
  const float* __restrict__ cellE;
  LayerTable L;
  double eta, epsilon, atcv;
  int atnum, hasCrackPressure;
  int unilateral;  // 1 = NOCOMPRESSION (VFCtx.unilateral)
  double hx, hy, hz;  // cell size (the tensor-product kernels)
};

// f (3N) = thermo-poro + crack-pressure load (VFMech.c:386-447, 533-589), so that
// F_U = K u - f.  Overwrites f.
// With E.unilateral the thermo-poro load depends on u0 through the sign of tr(eps(u0))
// (VF_GradientUThermoPoroNoCompression3D_local, VFMech.c:456-524); u0 = null reads as 0.
cudaError_t launch_u_rhs(const ElemArgs& E, const double* v, const double* theta,
                         const double* thetaRef, const double* p, double* f, cudaStream_t s,
                         const double* u0 = nullptr);
// d (3N) = diag K(v) (with E.unilateral: of K(v; u0)), Dirichlet rows 1.  Overwrites d.
cudaError_t launch_u_diag(const ElemArgs& E, const double* v, const uint8_t* bcbits, double* d,
                          cudaStream_t s, const double* u0 = nullptr);
// NOCOMPRESSION sign pattern: flags[cell] bit g = (tr(eps(u)) < 0 at Gauss point g).
cudaError_t launch_nc_flags(const ElemArgs& E, const double* u, uint32_t* flags, cudaStream_t s);
// coef (27 per cell in the vcoef_index layout: per element layer, 27 planes of the
// layer's cells, so that a tile's values are one box of a 3-D tensor copy) = w_g
// (2 W_g(u,theta) [+ Gc/(2c_w)/eps for AT2]) in FP64 and, if coef32 is not null, FP32.
cudaError_t launch_v_coef(const ElemArgs& E, const double* u, const double* theta,
                          const double* thetaRef, double* coef, float* coef32, cudaStream_t s);
// b (N) = AT linear term + crack pressure term (VFMech.c:2294-2384).  Overwrites b.
cudaError_t launch_v_rhs(const ElemArgs& E, const double* u, const double* p, double* b,
                         cudaStream_t s);
// d (N) = diag K_V.  Overwrites d.
cudaError_t launch_v_diag(const ElemArgs& E, const double* coef, double* d, cudaStream_t s);

// Energies: out[0] elastic, out[1] pressure work, out[2] surface, out[3] crack
// opening volume.  partial must hold 2*4*nblocks doubles; out is device memory.
int energy_blocks();
cudaError_t launch_energies(const ElemArgs& E, const double* u, const double* v,
                            const double* theta, const double* thetaRef, const double* p,
                            double* partial, double* out, double* cellcov, cudaStream_t s);

// In-situ boundary tractions (VFMech.c:598-715, 983-1102, 1196-1407, 1630-1848).
struct InsituArgs {
  int nx, ny, nz;
  double hx, hy, hz, lz;
  double smin[6], smax[6];  // Voigt s11 s22 s33 s23 s13 s12 at z = 0 and z = lz
  int freec[6][3];          // face X0 X1 Y0 Y1 Z0 Z1 x component: 1 = no Dirichlet BC there
};
// f += the consistent face load of the tractions (faces in the order X0..Z1).
cudaError_t launch_insitu_load(const InsituArgs& A, double* f, cudaStream_t s);
// out[0] = work of the tractions on u, with the reference's layers (X1/Y1/Z1 one node
// layer inside the box); partial: >= 6 * 64 doubles of device memory.
cudaError_t launch_insitu_work(const InsituArgs& A, const double* u, double* partial, double* out,
                               cudaStream_t s);

}  // namespace vfgpu
