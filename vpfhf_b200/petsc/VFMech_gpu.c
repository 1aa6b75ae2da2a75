/*
 * VFMech_gpu.c -- drop-in replacements of the mechanics entry points of VPFHF
 * (VFMech.h:21-24: VF_StepU, VF_StepV, VF_UEnergy3D, VF_VEnergy3D) and of the
 * flow-coupling boundary (VFPermfield.h: VolumetricCrackOpening, VolumetricFractureWellRate,
 * UpdateFractureWidth) that run on a B200 through the vfgpu C ABI (include/vfgpu.h).
 *
 * Build it into VPFHF instead of VFMech.c's versions of these four functions
 * (compile this file with -I<repo>/include, link libvfgpu.so, and drop the four
 * definitions from VFMech.c): the callers (VPFHF.c, VFCommon.c:1166-1231 and the
 * ValidationTests drivers) link unchanged.  One MPI rank per GPU problem: the
 * DMDA must not be distributed (comm size 1); in-situ tractions and
 * UNILATERAL_NOCOMPRESSION are passed on to the device problem.
 */
#include "petsc.h"
#include "VFCartFE.h"
#include "VFCommon.h"
#include "VFMech.h"
#include "VFPermfield.h"
#include "vfgpu.h"

/* one device problem per VFCtx (VFCtx is the application's singleton in practice) */
static vfgpu_ctx *gpu_ctx = NULL;
static const VFCtx *gpu_owner = NULL;

#define VFGPU_CHK(call)                                                           \
  do {                                                                            \
    int vfgpu_rc_ = (call);                                                       \
    if (vfgpu_rc_ < 0)                                                            \
      SETERRQ2(PETSC_COMM_SELF, PETSC_ERR_LIB, "%s: %s", #call, vfgpu_last_error()); \
  } while (0)

static void to_vfgpu_bc(const VFBC *in, vfgpu_bc *out) {
  int i;
  for (i = 0; i < 6; i++) {
    out->face[i] = (int)in->face[i];
    out->faceValue[i] = (double)in->faceValue[i];
  }
  for (i = 0; i < 8; i++) {
    out->vertex[i] = (int)in->vertex[i];
    out->vertexValue[i] = (double)in->vertexValue[i];
  }
}

/* Creates the device problem from the DMDA and the VFCtx the first time, and
 * refreshes material, phase-field parameters and BCs on every call (drivers
 * such as test18.c edit ctx->bcU between VFInitialize and the solves). */
static PetscErrorCode vfgpu_setup(VFCtx *ctx) {
  PetscErrorCode ierr;
  PetscMPIInt size;
  PetscInt nx, ny, nz, l, ek;
  PetscReal BBmin[3], BBmax[3];
  vfgpu_matprop mp[16];
  vfgpu_vfprop vf;
  vfgpu_bc bu[3], bv;
  int layer[4096];

  PetscFunctionBegin;
  ierr = MPI_Comm_size(PETSC_COMM_WORLD, &size);CHKERRQ(ierr);
  if (size != 1) SETERRQ(PETSC_COMM_WORLD, PETSC_ERR_SUP, "vfgpu: one rank per problem");
  if (ctx->nlayer > 16) SETERRQ(PETSC_COMM_WORLD, PETSC_ERR_SUP, "vfgpu: at most 16 layers");
  ierr = DMDAGetInfo(ctx->daVect, NULL, &nx, &ny, &nz, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                     NULL, NULL);CHKERRQ(ierr);
  if (nz - 1 > 4096) SETERRQ(PETSC_COMM_WORLD, PETSC_ERR_SUP, "vfgpu: at most 4097 planes");
  if (!gpu_ctx || gpu_owner != ctx) {
    vfgpu_grid g;
    if (gpu_ctx) vfgpu_destroy(gpu_ctx);
    ierr = DMDAGetBoundingBox(ctx->daVect, BBmin, BBmax);CHKERRQ(ierr);
    g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
    g.lx = BBmax[0] - BBmin[0]; g.ly = BBmax[1] - BBmin[1]; g.lz = BBmax[2] - BBmin[2];
    VFGPU_CHK(vfgpu_create(&g, &gpu_ctx));
    gpu_owner = ctx;
  }
  for (l = 0; l < ctx->nlayer; l++) {
    mp[l].E = ctx->matprop[l].E;
    mp[l].nu = ctx->matprop[l].nu;
    mp[l].alpha = ctx->matprop[l].alpha;
    mp[l].beta = ctx->matprop[l].beta;
    mp[l].Gc = ctx->matprop[l].Gc;
  }
  for (ek = 0; ek < nz - 1; ek++) layer[ek] = (int)ctx->layer[ek];
  VFGPU_CHK(vfgpu_set_matprop(gpu_ctx, (int)ctx->nlayer, mp, layer));
  vf.epsilon = ctx->vfprop.epsilon;
  vf.eta = ctx->vfprop.eta;
  vf.irrevtol = ctx->vfprop.irrevtol;
  vf.atnum = (int)ctx->vfprop.atnum;
  vf.hasCrackPressure = ctx->hasCrackPressure ? 1 : 0;
  VFGPU_CHK(vfgpu_set_vfprop(gpu_ctx, &vf));
  for (l = 0; l < 3; l++) to_vfgpu_bc(&ctx->bcU[l], &bu[l]);
  to_vfgpu_bc(&ctx->bcV[0], &bv);
  VFGPU_CHK(vfgpu_set_bc(gpu_ctx, bu, &bv));
  {
    double smin[6], smax[6];
    for (l = 0; l < 6; l++) {
      smin[l] = ctx->insitumin[l];
      smax[l] = ctx->insitumax[l];
    }
    VFGPU_CHK(vfgpu_set_insitu(gpu_ctx, ctx->hasInsitu ? smin : NULL, smax));
  }
  VFGPU_CHK(vfgpu_set_unilateral(gpu_ctx, ctx->unilateral == UNILATERAL_NOCOMPRESSION
                                              ? VFGPU_UNILATERAL_NOCOMPRESSION
                                              : VFGPU_UNILATERAL_NONE));
  PetscFunctionReturn(0);
}

static PetscErrorCode push(Vec v, int field) {
  PetscErrorCode ierr;
  const PetscScalar *a;
  PetscFunctionBegin;
  ierr = VecGetArrayRead(v, &a);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_set_field(gpu_ctx, field, (const double *)a));
  ierr = VecRestoreArrayRead(v, &a);CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

static PetscErrorCode pull(Vec v, int field) {
  PetscErrorCode ierr;
  PetscScalar *a;
  PetscFunctionBegin;
  ierr = VecGetArray(v, &a);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_get_field(gpu_ctx, field, (double *)a));
  ierr = VecRestoreArray(v, &a);CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* The fields every solve reads through ctx->fields (VFMech.c:1505-1532, 2729-2758). */
static PetscErrorCode push_inputs(VFFields *fields) {
  PetscErrorCode ierr;
  PetscFunctionBegin;
  ierr = push(fields->U, VFGPU_FIELD_U);CHKERRQ(ierr);
  ierr = push(fields->V, VFGPU_FIELD_V);CHKERRQ(ierr);
  ierr = push(fields->VIrrev, VFGPU_FIELD_VIRREV);CHKERRQ(ierr);
  ierr = push(fields->BCU, VFGPU_FIELD_BCU);CHKERRQ(ierr);
  ierr = push(fields->theta, VFGPU_FIELD_THETA);CHKERRQ(ierr);
  ierr = push(fields->thetaRef, VFGPU_FIELD_THETAREF);CHKERRQ(ierr);
  ierr = push(fields->pressure, VFGPU_FIELD_PRESSURE);CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

static void solve_opts(vfgpu_solve_opts *o) {
  PetscBool flg;
  PetscInt prec = 0, pc = VFGPU_PC_JACOBI;
  vfgpu_default_solve_opts(o);
  /* -vfgpu_precision 0 (FP64, default) | 1 (FP32 inner solves + FP64 refinement) */
  PetscOptionsGetInt(NULL, NULL, "-vfgpu_precision", &prec, &flg);
  o->precision = (int)prec;
  /* -vfgpu_pc 0 (Jacobi, the reference's KSPCG+Jacobi, default) | 1 (multigrid V-cycle;
     same stopping test; needs >= 9 nodes along some axis) | 2 (multigrid on grids with
     >= 65 nodes along some axis, Jacobi below) */
  PetscOptionsGetInt(NULL, NULL, "-vfgpu_pc", &pc, &flg);
  o->pc = (int)pc;
}

PetscErrorCode VF_StepU(VFFields *fields, VFCtx *ctx) {
  PetscErrorCode ierr;
  vfgpu_solve_opts o;
  vfgpu_solve_stats st;
  int rc;
  PetscFunctionBegin;
  ierr = vfgpu_setup(ctx);CHKERRQ(ierr);
  ierr = push_inputs(fields);CHKERRQ(ierr);
  solve_opts(&o);
  rc = vfgpu_step_u(gpu_ctx, &o, &st);
  VFGPU_CHK(rc);
  ierr = pull(fields->U, VFGPU_FIELD_U);CHKERRQ(ierr);
  if (st.reason < 0) {
    ierr = PetscPrintf(PETSC_COMM_WORLD, "[ERROR] snesU diverged with reason %d\n", st.reason);CHKERRQ(ierr);
  } else {
    ierr = PetscPrintf(PETSC_COMM_WORLD, "      snesU converged in %d iterations %d.\n",
                       st.newton_its, st.reason);CHKERRQ(ierr);
  }
  PetscFunctionReturn(0);
}

PetscErrorCode VF_StepV(VFFields *fields, VFCtx *ctx) {
  PetscErrorCode ierr;
  vfgpu_solve_opts o;
  vfgpu_solve_stats st;
  PetscReal vmin, vmax;
  int rc;
  PetscFunctionBegin;
  ierr = vfgpu_setup(ctx);CHKERRQ(ierr);
  ierr = push_inputs(fields);CHKERRQ(ierr);
  solve_opts(&o);
  rc = vfgpu_step_v(gpu_ctx, &o, &st);
  VFGPU_CHK(rc);
  ierr = pull(fields->V, VFGPU_FIELD_V);CHKERRQ(ierr);
  if (st.reason < 0) {
    ierr = PetscPrintf(PETSC_COMM_WORLD, "[ERROR] snesV diverged with reason %d\n", st.reason);CHKERRQ(ierr);
  } else {
    ierr = PetscPrintf(PETSC_COMM_WORLD, "      snesV converged in %d iterations %d.\n",
                       st.newton_its, st.reason);CHKERRQ(ierr);
  }
  ierr = VecMin(fields->V, NULL, &vmin);CHKERRQ(ierr);
  ierr = VecMax(fields->V, NULL, &vmax);CHKERRQ(ierr);
  ierr = PetscPrintf(PETSC_COMM_WORLD, "      V min / max:     %e %e\n", vmin, vmax);CHKERRQ(ierr);
  PetscFunctionReturn(st.reason < 0 ? st.reason : 0);  /* as VFMech.c:3070-3081 */
}

PetscErrorCode VF_UEnergy3D(PetscReal *ElasticEnergy, PetscReal *InsituWork,
                            PetscReal *PressureWork, Vec U, VFCtx *ctx) {
  PetscErrorCode ierr;
  double el, iw, pw;
  PetscFunctionBegin;
  ierr = vfgpu_setup(ctx);CHKERRQ(ierr);
  ierr = push_inputs(ctx->fields);CHKERRQ(ierr);
  ierr = push(U, VFGPU_FIELD_U);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_u_energy(gpu_ctx, &el, &iw, &pw));
  *ElasticEnergy = el;
  *InsituWork = iw;
  *PressureWork = pw;
  PetscFunctionReturn(0);
}

PetscErrorCode VF_VEnergy3D(PetscReal *SurfaceEnergy, VFFields *fields, VFCtx *ctx) {
  PetscErrorCode ierr;
  double s;
  PetscFunctionBegin;
  ierr = vfgpu_setup(ctx);CHKERRQ(ierr);
  ierr = push(fields->V, VFGPU_FIELD_V);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_v_energy(gpu_ctx, &s));
  *SurfaceEnergy = s;
  PetscFunctionReturn(0);
}

/* ---- flow-coupling boundary: drop-in replacements of VFPermfield.h:32 and :36 (build
 * them instead of VFPermfield.c's versions).  fields->widthc and fields->pmult are cell
 * vectors (daScalCell), fields->width a node vector (daScal), as UpdateFractureWidth
 * fills them (VFPermfield.c:267-562). ---- */
PetscErrorCode UpdateFractureWidth(VFCtx *ctx, VFFields *fields) {
  PetscErrorCode ierr;
  PetscScalar *wc, *wn, *pm;
  vfgpu_width_opts o;
  int nstall = 0;
  PetscFunctionBegin;
  ierr = vfgpu_setup(ctx);CHKERRQ(ierr);
  ierr = push(fields->U, VFGPU_FIELD_U);CHKERRQ(ierr);
  ierr = push(fields->V, VFGPU_FIELD_V);CHKERRQ(ierr);
  vfgpu_default_width_opts(&o);
  o.int_length = ctx->WidthIntLenght;
  o.width_tol = ctx->width_tol;
  o.remove_tip_effect = ctx->removeTipEffect ? 1 : 0;
  ierr = VecGetArray(fields->widthc, &wc);CHKERRQ(ierr);
  ierr = VecGetArray(fields->width, &wn);CHKERRQ(ierr);
  ierr = VecGetArray(fields->pmult, &pm);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_update_fracture_width(gpu_ctx, &o, (double *)wc, (double *)wn, (double *)pm,
                                        &nstall));
  ierr = VecRestoreArray(fields->pmult, &pm);CHKERRQ(ierr);
  ierr = VecRestoreArray(fields->width, &wn);CHKERRQ(ierr);
  ierr = VecRestoreArray(fields->widthc, &wc);CHKERRQ(ierr);
  if (nstall) {
    ierr = PetscPrintf(PETSC_COMM_WORLD,
                       "      vfgpu: %d band cells with zero grad V at the centre kept width 0\n",
                       nstall);CHKERRQ(ierr);
  }
  PetscFunctionReturn(0);
}

/* VolumetricCrackOpening (VFPermfield.c:75-152): the total and fields->VolCrackOpening,
 * the node average of the per-cell opening. */
PetscErrorCode VolumetricCrackOpening(PetscReal *CrackVolume, VFCtx *ctx, VFFields *fields) {
  PetscErrorCode ierr;
  PetscInt nx, ny, nz;
  PetscScalar *nodev;
  double cov = 0., *cellv = NULL;
  PetscFunctionBegin;
  ierr = vfgpu_setup(ctx);CHKERRQ(ierr);
  ierr = push(fields->U, VFGPU_FIELD_U);CHKERRQ(ierr);
  ierr = push(fields->V, VFGPU_FIELD_V);CHKERRQ(ierr);
  ierr = DMDAGetInfo(ctx->daVect, NULL, &nx, &ny, &nz, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                     NULL, NULL);CHKERRQ(ierr);
  ierr = PetscMalloc((size_t)(nx - 1) * (ny - 1) * (nz - 1) * sizeof(double), &cellv);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_crack_opening(gpu_ctx, &cov, cellv));
  ierr = VecGetArray(fields->VolCrackOpening, &nodev);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_cell_to_node(gpu_ctx, cellv, (double *)nodev));
  ierr = VecRestoreArray(fields->VolCrackOpening, &nodev);CHKERRQ(ierr);
  ierr = PetscFree(cellv);CHKERRQ(ierr);
  *CrackVolume = cov;
  PetscFunctionReturn(0);
}

PetscErrorCode VolumetricFractureWellRate(PetscReal *InjectedVolume, VFCtx *ctx, VFFields *fields) {
  PetscErrorCode ierr;
  const PetscScalar *r;
  double rate = 0.;
  PetscFunctionBegin;
  ierr = vfgpu_setup(ctx);CHKERRQ(ierr);
  ierr = push(fields->V, VFGPU_FIELD_V);CHKERRQ(ierr);
  ierr = VecGetArrayRead(ctx->RegFracWellFlowRate, &r);CHKERRQ(ierr);
  VFGPU_CHK(vfgpu_fracture_well_rate(gpu_ctx, (const double *)r, &rate));
  ierr = VecRestoreArrayRead(ctx->RegFracWellFlowRate, &r);CHKERRQ(ierr);
  *InjectedVolume = rate;
  PetscFunctionReturn(0);
}
