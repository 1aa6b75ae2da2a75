/*
 * vfgpu.h -- C ABI of the B200 implementation of VPFHF's alternate-minimisation
 * hot path (U = displacement, V = phase field).  Plain C types only.
 *
 * One vfgpu_ctx holds one problem resident on the GPU that was current when
 * it was created: the grid, the per-layer material, the phase-field
 * parameters, the Dirichlet BCs and the fields (U, V, VIrrev, BCU, theta,
 * thetaRef, pressure).  It mirrors what the reference keeps in VFCtx /
 * VFFields (VFCommon.h:35-63, 69-90, 213-380).  All arrays are in the DMDA
 * natural ordering (x fastest, then y, then z); U-like arrays interlace the 3
 * components (u[3*node + c]).  Array arguments may be host or device pointers
 * (device pointers of the ctx's GPU are used in place).
 *
 * Every function returns an int status: VFGPU_OK (0), > 0 for a solver that
 * stopped without converging, < 0 for an error; vfgpu_last_error() gives the
 * message of the last failure on the calling thread.  No exception crosses the
 * ABI.  Calls on one ctx must not overlap; different ctxs are independent.
 */
#ifndef VFGPU_H
#define VFGPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vfgpu_ctx vfgpu_ctx;

/* status codes */
#define VFGPU_OK 0
#define VFGPU_NOT_CONVERGED 1 /* solver hit its iteration cap                 */
#define VFGPU_DIVERGED 2      /* solver diverged (NaN, indefinite, dtol)       */
#define VFGPU_ERR_INVALID -1  /* bad argument                                  */
#define VFGPU_ERR_CUDA -2     /* CUDA runtime error                            */
#define VFGPU_ERR_OOM -3      /* device allocation failed                      */
#define VFGPU_ERR_STATE -4    /* ctx not ready (missing material, fields ...)   */

/* arithmetic of the operator applications / inner Krylov solves */
#define VFGPU_FP64 0   /* everything in FP64 (the reference's PetscReal)       */
#define VFGPU_MIXED 1  /* FP32 operator inside FP64 iterative refinement       */

/* BC types -- same numbering as the reference's BCTYPE (VFCartFE.h:95-100) */
#define VFGPU_BC_NONE 0
#define VFGPU_BC_ZERO 1
#define VFGPU_BC_ONE 2
#define VFGPU_BC_FIXED 3

/* fields (VFFields members used by the hot path) */
#define VFGPU_FIELD_U 0        /* 3N displacement                                  */
#define VFGPU_FIELD_V 1        /* N phase field                                    */
#define VFGPU_FIELD_VIRREV 2   /* N irreversibility reference / AT1 upper bound     */
#define VFGPU_FIELD_BCU 3      /* 3N boundary displacement (FIXED Dirichlet values) */
#define VFGPU_FIELD_THETA 4    /* N temperature                                    */
#define VFGPU_FIELD_THETAREF 5 /* N reference temperature                          */
#define VFGPU_FIELD_PRESSURE 6 /* N pore / crack pressure (one Vec, quirk Q5)       */

typedef struct {
  int nx, ny, nz;       /* nodes per axis (-n)                                 */
  double lx, ly, lz;    /* box lengths (-l); X[i] = i*lx/(nx-1)               */
} vfgpu_grid;

/* subset of VFMatProp (VFCommon.h:69-80) used by the mechanics */
typedef struct {
  double E, nu;   /* Young's modulus, Poisson ratio (lambda, mu as VFMatPropGet) */
  double alpha;   /* linear thermal expansion                                    */
  double beta;    /* Biot coefficient                                            */
  double Gc;      /* fracture toughness                                          */
} vfgpu_matprop;

/* subset of VFProp (VFCommon.h:170-179) */
typedef struct {
  double epsilon, eta, irrevtol;
  int atnum;            /* 1 = AT1, 2 = AT2                                     */
  int hasCrackPressure; /* VFCtx.hasCrackPressure (-pressurize)                 */
} vfgpu_vfprop;

/* VFBC (VFCartFE.h:137-144) without the unused edge entries */
typedef struct {
  int face[6];           /* X0,X1,Y0,Y1,Z0,Z1: VFGPU_BC_*                          */
  double faceValue[6];
  int vertex[8];         /* X0Y0Z0,X1Y0Z0,X0Y1Z0,X1Y1Z0,X0Y0Z1,X1Y0Z1,X0Y1Z1,X1Y1Z1 */
  double vertexValue[8];
} vfgpu_bc;

/* Message of the last failed call on this thread ("" if none). */
const char* vfgpu_last_error(void);

/* Creates a ctx on the current CUDA device.  Replaces the DMDA/Vec set-up of
 * VFGeometryInitialize + VFFieldsInitialize (VFCommon.c:277-451, 629-857):
 * U = 0, V = VIrrev = 1, theta = thetaRef = pressure = 0. */
int vfgpu_create(const vfgpu_grid* grid, vfgpu_ctx** out);
int vfgpu_destroy(vfgpu_ctx* ctx);

/* Per-layer material (VFMatPropGet, VFCommon.c:506-588); layer[ek] for the
 * nz-1 element layers (VFLayerInit, VFCommon.c:1099-1120), NULL = all layer 0. */
int vfgpu_set_matprop(vfgpu_ctx* ctx, int nlayer, const vfgpu_matprop* mp, const int* layer);
/* Optional per-cell Young's modulus ((nx-1)(ny-1)(nz-1), NULL to clear); nu, alpha,
 * beta, Gc stay per layer.  Not a reference feature: the reference's material
 * is per layer only (VFCommon.h:79, "change them to Vec later"). */
int vfgpu_set_cell_modulus(vfgpu_ctx* ctx, const double* cellE);
int vfgpu_set_vfprop(vfgpu_ctx* ctx, const vfgpu_vfprop* vf);
/* ctx->bcU[3], ctx->bcV[1] (VFBCSetFromOptions, VFCartFE.c:1506-1574). */
int vfgpu_set_bc(vfgpu_ctx* ctx, const vfgpu_bc bcU[3], const vfgpu_bc* bcV);

int vfgpu_set_field(vfgpu_ctx* ctx, int field, const double* data);
int vfgpu_get_field(vfgpu_ctx* ctx, int field, double* data);

/* y = J_U x: the U Jacobian K(V) of VF_UIJacobian (VFMech.c:1897-2029) applied
 * matrix-free, Dirichlet rows identity (MatApplyDirichletBC, VFCartFE.c:1147-1296),
 * with the resident V.  x, y: 3N.  precision: VFGPU_FP64 or VFGPU_MIXED (FP32
 * kernel; x is rounded to FP32, y returned in FP64). */
int vfgpu_u_apply(vfgpu_ctx* ctx, int precision, const double* x, double* y);

#ifdef __cplusplus
}
#endif
#endif /* VFGPU_H */
