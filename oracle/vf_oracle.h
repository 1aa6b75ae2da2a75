/*
 * vf_oracle.h -- CPU oracle for the VPFHF alternate-minimisation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of the
 * reference's arithmetic (VFCartFE.c, VFMech.c, VFCracks.c, VFPermfield.c,
 * VFCommon.c of bourdin/VPFHF).  It is used by tests/ as the checker, by
 * __graft_entry__.smoke() as the checker and by bench.py as the timed CPU
 * baseline.  The product (vpfhf_b200/, libvfgpu.so) never links or calls it.
 *
 * Parity pinning: the restatement is checked against the reference's own
 * known-answer content (ValidationTests/results/runtest1.out energies, the
 * analytic 1-D bar energy 0.2 t^2, Clapeyron W_p = 2 E_el from
 * results/runtest8.out / runtest9.out) -- see tests/test_oracle_*.py.
 * PETSc itself is not available, so iteration-level parity with PETSc's
 * SNES/KSP is not pinned; converged solutions are (the U problem is SPD and
 * the V problem is a strictly convex box-constrained QP, so both have unique
 * solutions that any converged solver reproduces within its tolerance).
 *
 * Layout conventions (DMDA natural ordering, x fastest):
 *   node(i,j,k)      = (k*ny + j)*nx + i
 *   U dof (node,c)   = 3*node + c          (interlaced, c = 0,1,2)
 *   cell(ei,ej,ek)   = (ek*(ny-1) + ej)*(nx-1) + ei
 *   local node a of a cell = i + 2*j + 4*k  (i,j,k in {0,1}),
 *   which is the reference's (k,j,i) lexicographic order (VFMech.c:1581-1588).
 */
#ifndef VF_ORACLE_H
#define VF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VFO_MAXLAYER 16

/* BC types, same numbering as the reference's BCTYPE (VFCartFE.h:95-100). */
enum { VFO_NONE = 0, VFO_ZERO = 1, VFO_ONE = 2, VFO_FIXED = 3 };

typedef struct {
  int    nx, ny, nz;            /* nodes per axis                                   */
  double lx, ly, lz;            /* box lengths (coordinates X[i] = i*lx/(nx-1))      */
  int    nlayer;                /* material layers (VFCommon.h:296 matprop[])        */
  double E[VFO_MAXLAYER], nu[VFO_MAXLAYER];
  double alpha[VFO_MAXLAYER];   /* thermal expansion (VFCommon.h:72)                  */
  double beta[VFO_MAXLAYER];    /* Biot coefficient  (VFCommon.h:74)                  */
  double Gc[VFO_MAXLAYER];
  const int    *layer;          /* nz-1 entries: layer of element layer ek, or NULL   */
  const double *cellE;          /* optional per-cell Young's modulus (generalisation) */
  double epsilon, eta, irrevtol;
  int    atnum;                 /* 1 = AT1, 2 = AT2                                   */
  int    hasCrackPressure;
  int    nthreads;              /* OpenMP threads for the fast variants (0 = default) */
  /* in-situ stresses (VFCommon.c:132-149): Voigt s11 s22 s33 s23 s13 s12 at z = 0
   * (min) and z = lz (max), linear in z between; insitu_free[face][c] = 1 where
   * bcU[c].face[face] == NONE (faces X0 X1 Y0 Y1 Z0 Z1) */
  int    hasInsitu;
  double insitumin[6], insitumax[6];
  int    insitu_free[6][3];
  /* VFCtx.unilateral (VFCommon.c:176-177): 0 = UNILATERAL_NONE, 1 = NOCOMPRESSION --
   * the spherical part of the energy is not degraded where tr(eps(u)) < 0
   * (UNILATERAL_THRES = 0, VFMech.c:6), which makes the U residual depend on U */
  int    unilateral;
} vfo_problem;

typedef struct {
  double rtol, atol, dtol;      /* KSP tolerances (VFCommon.c:1039)                   */
  int    maxit;
  double snes_rtol, snes_atol, snes_stol;
  int    snes_maxit;
} vfo_solver_opts;

typedef struct {
  int    newton_its;            /* SNES iterations                                    */
  int    ksp_its;               /* total KSP iterations                               */
  int    reason;                /* SNES converged reason (PETSc numbering)            */
  double fnorm0, fnorm;
} vfo_stats;

/* ---- element tables: VFCartFEElement3DInit (VFCartFE.c:216-269) ---- */
int vfo_tables(double hx, double hy, double hz,
               double w[27], double phi[8 * 27], double dphi[8 * 3 * 27]);

/* ---- Dirichlet BC: VecApplyDirichletBC precedence (VFCartFE.c:493-738) ----
 * face: dof*6 BCTYPE, vertex: dof*8 BCTYPE (VERTEX enum order, VFCartFE.h:121-130),
 * bcu: FIXED values per dof (dof*N) or NULL.  Outputs mask[dof*N] and value[dof*N]. */
int vfo_bc_build(int nx, int ny, int nz, int dof, const int *face, const int *vertex,
                 const double *bcu, uint8_t *mask, double *value);

/* ---- U operator (VFMech.c:227-290, 1456-1887) ---- */
int vfo_u_element_matrix(const vfo_problem *P, int ei, int ej, int ek, const double *v,
                         double K[576]);
int vfo_u_apply_ref(const vfo_problem *P, const double *v, const double *x,
                    const uint8_t *bcmask, double *y);
int vfo_u_apply_mf(const vfo_problem *P, const double *v, const double *x,
                   const uint8_t *bcmask, double *y);
int vfo_u_rhs(const vfo_problem *P, const double *v, const double *theta,
              const double *thetaRef, const double *p, double *f);
int vfo_u_residual_ref(const vfo_problem *P, const double *u, const double *v,
                       const double *theta, const double *thetaRef, const double *p,
                       const uint8_t *bcmask, const double *bcval, double *F);
int vfo_u_diag(const vfo_problem *P, const double *v, const uint8_t *bcmask, double *d);
/* NOCOMPRESSION forms need the displacement u0 that fixes the sign of tr(eps) at each
 * Gauss point (VF_BilinearFormUNoCompression3D_local, VFMech.c:299-376, and
 * VF_GradientUThermoPoroNoCompression3D_local, VFMech.c:456-524); with
 * unilateral = 0, or u0 = NULL (tr = 0: the tensile branch), they equal the
 * functions above. */
int vfo_u_apply_mf_u(const vfo_problem *P, const double *u0, const double *v, const double *x,
                     const uint8_t *bcmask, double *y);
int vfo_u_apply_ref_u(const vfo_problem *P, const double *u0, const double *v, const double *x,
                      const uint8_t *bcmask, double *y);
int vfo_u_rhs_u(const vfo_problem *P, const double *u0, const double *v, const double *theta,
                const double *thetaRef, const double *p, double *f);
int vfo_u_diag_u(const vfo_problem *P, const double *u0, const double *v, const uint8_t *bcmask,
                 double *d);
/* CSR assembly of K(v) with BC rows -> identity (VF_UIJacobian, VFMech.c:1897-2029). */
int64_t vfo_u_csr_nnz(const vfo_problem *P);
int vfo_u_assemble_csr(const vfo_problem *P, const double *v, const uint8_t *bcmask,
                       int64_t *rowptr, int32_t *colidx, double *vals);
int vfo_csr_spmv(int64_t nrows, const int64_t *rowptr, const int32_t *colidx,
                 const double *vals, const double *x, double *y, int nthreads);

/* ---- V operator (VFMech.c:2032-2153, 2287-2384, 2687-3029) ---- */
int vfo_v_element_matrix(const vfo_problem *P, int ei, int ej, int ek, const double *u,
                         const double *theta, const double *thetaRef, double K[64]);
int vfo_v_rhs(const vfo_problem *P, const double *u, const double *p, double *b);
int vfo_v_residual_ref(const vfo_problem *P, const double *u, const double *v,
                       const double *theta, const double *thetaRef, const double *p,
                       const double *virrev, const uint8_t *bcmask, const double *bcval,
                       double *F);
/* J_V x with BC rows+cols and (AT2) irreversibility rows+cols -> identity. */
int vfo_v_apply(const vfo_problem *P, const double *u, const double *theta,
                const double *thetaRef, const double *virrev, const uint8_t *bcmask,
                const double *x, double *y);
int vfo_v_diag(const vfo_problem *P, const double *u, const double *theta,
               const double *thetaRef, const double *virrev, const uint8_t *bcmask,
               double *d);

/* ---- energies and crack opening (VFMech.c:725-974, 2394-2526; VFPermfield.c:15-152) ---- */
int vfo_u_energy(const vfo_problem *P, const double *u, const double *v,
                 const double *theta, const double *thetaRef, const double *p,
                 double out[2] /* elastic, pressure work */);
int vfo_v_energy(const vfo_problem *P, const double *v, double *surface);
int vfo_cov(const vfo_problem *P, const double *u, const double *v, double *cov,
            double *cellcov /* (nx-1)(ny-1)(nz-1) or NULL */);

/* ---- in-situ boundary tractions (VFMech.c:598-715, 983-1102, 1196-1407, 1630-1848) ----
 * Work of the tractions on U, with the reference's layer choice for the X1/Y1/Z1
 * faces (the cell layer before the last, so the node layer one inside the box). */
int vfo_insitu_work(const vfo_problem *P, const double *u, double *work);

/* ---- flow-coupling boundary (VFPermfield.c, VFCommon.c:897-914) ----
 * vfo_width_int_length: VFCtx.WidthIntLenght.  vfo_fracture_width: UpdateFractureWidth
 * (VFPermfield.c:267-562) -- widthc and pmult per cell; nstall counts band cells whose
 * march cannot advance (zero grad V at the centre: the reference loops there forever).
 * vfo_cell_to_node: CellToNodeInterpolation (VFPermfield.c:1156-1330), volume-weighted.
 * vfo_fracture_well_rate: VolumetricFractureWellRate (VFPermfield.c:1513-1604). */
double vfo_width_int_length(const vfo_problem *P);
int vfo_fracture_width(const vfo_problem *P, const double *u, const double *v, double L,
                       double width_tol, int remove_tip, double *widthc, double *pmult,
                       int *nstall);
int vfo_cell_to_node(const vfo_problem *P, const double *cellv, double *nodev);
int vfo_fracture_well_rate(const vfo_problem *P, const double *v, const double *regrate,
                           double *rate);

/* ---- penny crack initial V (VFCracks.c:101-227) ---- */
int vfo_penny_crack_v(const vfo_problem *P, const double center[3], double r,
                      double theta_deg, double phi_deg, double thickness, double *v);
/* rectangular crack (VFCracks.c:331-513) and the several-crack minimum (VFCommon.c:823-857) */
double vfo_rect_distance(const double x[3], const double corners[9]);
int vfo_rect_crack_v(const vfo_problem *P, const double corners[9], double thickness, double *v);
int vfo_cracks_v(const vfo_problem *P, int npenny, const double *penny, int nrect,
                 const double *rect, double *v);

/* ---- solvers (PETSc semantics restated: VFCommon.c:1005-1088) ---- */
int vfo_step_u(const vfo_problem *P, double *u, const double *v, const double *theta,
               const double *thetaRef, const double *p, const uint8_t *bcmask,
               const double *bcval, const vfo_solver_opts *o, vfo_stats *st);
int vfo_step_v(const vfo_problem *P, double *v, const double *u, const double *theta,
               const double *thetaRef, const double *p, const double *virrev,
               const double *lb, const double *ub, const uint8_t *bcmask,
               const double *bcval, const vfo_solver_opts *o, vfo_stats *st);

/* The same two solves by the reference's method, for the timed CPU AM-step baseline:
 * residuals from re-formed element matrices, the Jacobian assembled into CSR at every
 * Newton iteration, KSPCG + Jacobi on the assembled matrix (VFMech.c:1555-1596,
 * 1897-2029, 2772-2848, 2948-3027); element loops and vector sums on all threads.
 * *seconds_assembly = time spent assembling the Jacobians.  UNILATERAL_NONE only. */
int vfo_step_u_asm(const vfo_problem *P, double *u, const double *v, const double *theta,
                   const double *thetaRef, const double *p, const uint8_t *bcmask,
                   const double *bcval, const vfo_solver_opts *o, vfo_stats *st,
                   double *seconds_assembly);
int vfo_step_v_asm(const vfo_problem *P, double *v, const double *u, const double *theta,
                   const double *thetaRef, const double *p, const double *virrev,
                   const double *lb, const double *ub, const uint8_t *bcmask,
                   const double *bcval, const vfo_solver_opts *o, vfo_stats *st,
                   double *seconds_assembly);

#ifdef __cplusplus
}
#endif
#endif
