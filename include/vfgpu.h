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

/* Solver options.  Defaults (vfgpu_default_solve_opts) are the reference's:
 * SNES atol = rtol = stol = 1e-8 (VFCommon.c:1024, 1071), KSPCG rtol 1e-8,
 * atol 1e-10 (VFCommon.c:1039, 1081) with a Jacobi preconditioner. */
typedef struct {
  int precision;          /* VFGPU_FP64 or VFGPU_MIXED                                  */
  double ksp_rtol, ksp_atol, ksp_dtol;
  int ksp_maxit;          /* per linear solve (per inner solve for VFGPU_MIXED)         */
  double snes_rtol, snes_atol, snes_stol;
  int snes_maxit;
  double inner_rtol;      /* VFGPU_MIXED: relative tolerance of each FP32 inner solve   */
  int max_refine;         /* VFGPU_MIXED: cap on FP64 refinement steps per Newton step  */
  double time_limit;      /* wall-clock watchdog in seconds (0 = none)                  */
  int pc;                 /* StepU preconditioner: VFGPU_PC_JACOBI (the reference's) or  */
                          /* VFGPU_PC_MG (geometric multigrid V-cycle, FP32 under       */
                          /* VFGPU_MIXED, FP64 otherwise; FP64 CG with the Jacobi       */
                          /* solve's stopping test; needs >= 9 nodes along some axis)   */
                          /* or VFGPU_PC_AUTO (multigrid on grids with at least         */
                          /* VFGPU_PC_AUTO_MG_NODES nodes along some axis, else Jacobi) */
} vfgpu_solve_opts;

#define VFGPU_PC_JACOBI 0
#define VFGPU_PC_MG 1
#define VFGPU_PC_AUTO 2
#define VFGPU_PC_AUTO_MG_NODES 65

typedef struct {
  int newton_its;         /* SNES iterations                                            */
  int ksp_its;            /* total CG iterations (all inner solves)                     */
  int refine_its;         /* VFGPU_MIXED: FP64 refinement steps                         */
  int reason;             /* SNESConvergedReason numbering; -100 = watchdog             */
  double fnorm0, fnorm;   /* residual norm before / after (inactive-set norm for V)     */
  double seconds;
} vfgpu_solve_stats;

/* Message of the last failed call on this thread ("" if none). */
const char* vfgpu_last_error(void);

/* Creates a ctx on the current CUDA device.  Replaces the DMDA/Vec set-up of
 * VFGeometryInitialize + VFFieldsInitialize (VFCommon.c:277-451, 629-857):
 * U = 0, V = VIrrev = 1, theta = thetaRef = pressure = 0. */
int vfgpu_create(const vfgpu_grid* grid, vfgpu_ctx** out);
int vfgpu_destroy(vfgpu_ctx* ctx);

/* Device bytes a ctx of this grid holds once it has solved (fields + solver work
 * space); no counterpart in the reference.  Used for memory-based admission of
 * problems in the serving loop. */
int vfgpu_memory_estimate(const vfgpu_grid* grid, long long* bytes);

/* The multigrid hierarchy a solve with pc = VFGPU_PC_MG builds for this grid (host
 * only, no counterpart in the reference): *nlevels levels (1: the grid cannot be
 * coarsened and such a solve is refused), their node counts in dims[3 l .. 3 l + 2]
 * for l < min(*nlevels, max_levels), and the extra device bytes of the hierarchy in
 * precision `bytes` (8: FP64 V-cycle, 4: the FP32 one of VFGPU_MIXED) in *mg_bytes
 * (may be NULL). */
int vfgpu_mg_hierarchy(const vfgpu_grid* grid, int bytes, int max_levels, int* dims, int* nlevels,
                       long long* mg_bytes);

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

/* Unilateral model (-unilateral, VFCommon.c:176-177; VFUnilateralType).  With
 * NOCOMPRESSION the spherical part of the elastic energy is not degraded at Gauss
 * points where tr(eps(U)) < 0 (UNILATERAL_THRES = 0, VFMech.c:6): the U operator
 * (VFMech.c:299-376), thermo-poro load (456-524), elastic energy (819-908) and the
 * V coupling (2125-2153) switch per Gauss point, and StepU's Newton iterations
 * re-form operator, load and Jacobi diagonal at every iterate.  vfgpu_u_apply then
 * applies K(V; U) linearised at the resident U. */
#define VFGPU_UNILATERAL_NONE 0
#define VFGPU_UNILATERAL_NOCOMPRESSION 1
int vfgpu_set_unilateral(vfgpu_ctx* ctx, int type);

/* How the ctx's U applies split their work (no reference counterpart: a launch-shape
 * choice with bit-identical results).  ON: two waves -- the (tile, plane) units whose
 * elements all have a constant nodal phase field on a kernel with the fixed-weight element
 * alone, the rest on the general one; OFF: one wave over all units; AUTO (the default):
 * ON from a grid size per precision where it measured faster.  Grids with more than 2048
 * 32 x 8 element tiles per plane and NOCOMPRESSION always take one wave. */
#define VFGPU_U_SPLIT_AUTO 0
#define VFGPU_U_SPLIT_OFF 1
#define VFGPU_U_SPLIT_ON 2
int vfgpu_set_u_split(vfgpu_ctx* ctx, int mode);

/* In-situ stresses (-insitumin / -insitumax, VFCommon.c:132-149): Voigt
 * (s11, s22, s33, s23, s13, s12) at z = 0 and z = lz, linear in z between;
 * insitumax NULL = insitumin; insitumin NULL switches them off (hasInsitu).
 * Their tractions sigma.n load every boundary face component without a Dirichlet
 * BC (VF_UResidual, VFMech.c:1630-1848) and their work is the in-situ term of
 * vfgpu_u_energy (VFMech.c:1238-1407, with the reference's choice of the node
 * layer one inside the box for the X1/Y1/Z1 faces).  Where a component has a
 * Dirichlet BC on a face, no traction is used for it there; the reference's work
 * sum reuses the value another face wrote at a shared edge node instead. */
int vfgpu_set_insitu(vfgpu_ctx* ctx, const double insitumin[6], const double insitumax[6]);

int vfgpu_set_field(vfgpu_ctx* ctx, int field, const double* data);
int vfgpu_get_field(vfgpu_ctx* ctx, int field, double* data);

/* y = J_U x: the U Jacobian K(V) of VF_UIJacobian (VFMech.c:1897-2029) applied
 * matrix-free, Dirichlet rows identity (MatApplyDirichletBC, VFCartFE.c:1147-1296),
 * with the resident V.  x, y: 3N.  precision: VFGPU_FP64 or VFGPU_MIXED (FP32
 * kernel; x is rounded to FP32, y returned in FP64). */
int vfgpu_u_apply(vfgpu_ctx* ctx, int precision, const double* x, double* y);

/* Stream-ordered variant for device-resident data: x, y are device arrays of
 * the precision's type (double for VFGPU_FP64, float for VFGPU_MIXED); the
 * work is queued on the ctx's stream and the call returns without waiting. */
int vfgpu_u_apply_dev(vfgpu_ctx* ctx, int precision, const void* x, void* y);

/* The cudaStream_t every call of this ctx runs on (for event timing / ordering). */
int vfgpu_get_stream(vfgpu_ctx* ctx, void** stream);

void vfgpu_default_solve_opts(vfgpu_solve_opts* opts);

/* VF_StepU (VFMech.c:1436-1452): SNESSolve(snesU) on the resident U with the
 * resident V, theta, thetaRef, pressure; Newton + L2 line search, PCG(Jacobi),
 * the residual of VF_UResidual (VFMech.c:1456-1887).
 * Returns VFGPU_OK when converged, VFGPU_NOT_CONVERGED (iteration cap or
 * watchdog) or VFGPU_DIVERGED; the reference's VF_StepU returns 0 in all three
 * cases and only prints (VFMech.c:1445-1450).  opts may be NULL (defaults). */
int vfgpu_step_u(vfgpu_ctx* ctx, const vfgpu_solve_opts* opts, vfgpu_solve_stats* stats);

/* VF_StepV (VFMech.c:3057-3082): SNESSolve(snesV) with SNESVINEWTONRSLS on the
 * resident V: bounds [0,1] (AT2) or [0,VIrrev] (AT1, VFCommon.c:1149-1154),
 * residual of VF_VResidual (VFMech.c:2687-2879, thermo-poro term discarded as in
 * the reference), AT2 irreversibility where VIrrev <= irrevtol. */
int vfgpu_step_v(vfgpu_ctx* ctx, const vfgpu_solve_opts* opts, vfgpu_solve_stats* stats);

/* VFTimeStepPrepare (VFCommon.c:1132-1157): VIrrev := V; Dirichlet values into U
 * (from BCU for FIXED) and V. */
int vfgpu_time_step_prepare(vfgpu_ctx* ctx);

/* One alternate-minimisation iteration (VFCommon.c:1183-1202 loop body):
 * StepU, StepV, errV = ||V - Vold||_inf. */
int vfgpu_am_step(vfgpu_ctx* ctx, const vfgpu_solve_opts* opts, double* errV,
                  vfgpu_solve_stats* statsU, vfgpu_solve_stats* statsV);

/* VF_UEnergy3D (VFMech.c:1111-1427): elastic energy, in-situ work (0 unless
 * vfgpu_set_insitu) and pressure work. */
int vfgpu_u_energy(vfgpu_ctx* ctx, double* elastic, double* insitu, double* pressurework);
/* VF_VEnergy3D (VFMech.c:2474-2526): AT1/AT2 surface energy. */
int vfgpu_v_energy(vfgpu_ctx* ctx, double* surface);
/* VolumetricCrackOpening (VFPermfield.c:75-152): total and, if cellcov is not
 * NULL, the per-cell average ((nx-1)(ny-1)(nz-1)). */
int vfgpu_crack_opening(vfgpu_ctx* ctx, double* cov, double* cellcov);

/* ---- flow-coupling boundary (what VPFHF.c:91-101 calls between VF_StepP and VF_StepU's
 * consumers; the flow solvers themselves stay with the host) ---- */
typedef struct {
  double int_length;      /* VFCtx.WidthIntLenght; <= 0: 3 res + 4 epsilon (VFCommon.c:897-914) */
  double width_tol;       /* VFCtx.width_tol (-widthremoval_tol, VFCommon.c:111; default 0.1)  */
  int remove_tip_effect;  /* VFCtx.removeTipEffect (-removetipeffect, VFCommon.c:108; 0)       */
} vfgpu_width_opts;
void vfgpu_default_width_opts(vfgpu_width_opts* opts);
/* UpdateFractureWidth (VFPermfield.c:267-562) at the resident U and V: fields->widthc
 * (cells), fields->width (nodes, CellToNodeInterpolation VFPermfield.c:1156-1330) and
 * fields->pmult (cells: 0 where the integrated grad V exceeds width_tol, else 1).
 * Each output is host or device memory, or NULL (the results stay resident either
 * way).  nstalled (may be NULL): band cells whose march cannot advance because grad V
 * vanishes at their centre (the reference's loop does not end there); they get width 0. */
int vfgpu_update_fracture_width(vfgpu_ctx* ctx, const vfgpu_width_opts* opts, double* widthc,
                                double* width, double* pmult, int* nstalled);
/* VolumetricFractureWellRate (VFPermfield.c:1552-1604): sum over cells of the nodal
 * rate field regrate (ctx->RegFracWellFlowRate; N, host or device) times |grad V|,
 * integrated with the 27-point rule. */
int vfgpu_fracture_well_rate(vfgpu_ctx* ctx, const double* regrate, double* rate);
/* CellToNodeInterpolation (VFPermfield.c:1156-1330) of a scalar cell field: each node
 * takes the volume-weighted mean of its cells (cellv: (nx-1)(ny-1)(nz-1), nodev: N; host
 * or device memory). */
int vfgpu_cell_to_node(vfgpu_ctx* ctx, const double* cellv, double* nodev);

/* The SNES residuals at the resident fields: VF_UResidual (3N) and VF_VResidual (N). */
int vfgpu_u_residual(vfgpu_ctx* ctx, double* F);
int vfgpu_v_residual(vfgpu_ctx* ctx, double* F);

/* ---- crack initialisers ------------------------------------------------------ */
/* VFPennyCrack (VFCracks.h): disk of radius r around center, normal
 * (cos theta sin phi, sin theta sin phi, cos phi) with the angles in degrees. */
typedef struct {
  double center[3];
  double r, theta, phi, thickness;
} vfgpu_penny;
/* VFRectangularCrack (VFCracks.h): corners P1 = corners[0..2], P2 = [3..5],
 * P3 = [6..8]; the fourth corner is P2 + P3 - P1. */
typedef struct {
  double corners[9];
  double thickness;
} vfgpu_rect;

/* The crack part of VFFieldsInitialize (VFCommon.c:823-857) on the device:
 * V = VIrrev = pointwise minimum over the penny cracks (VFPennyCrackBuildVAT1/2,
 * VFCracks.c:136-227) and the rectangular cracks (VFRectangularCrackBuildVAT1/2,
 * VFCracks.c:436-513) with the profile of the ctx's atnum and epsilon; 1 where
 * there are none.  Any number of cracks. */
int vfgpu_init_cracks(vfgpu_ctx* ctx, int npenny, const vfgpu_penny* penny, int nrect,
                      const vfgpu_rect* rect);

/* ---- serving: a request loop over independent problems ------------------------
 * No counterpart in the reference (one problem per process there).  A server owns
 * worker threads on one GPU.  Each request is a whole fracture problem: grid,
 * material, phase-field parameters, BCs, cracks, a uniform crack pressure and a
 * number of AM iterations.  Requests are admitted in arrival order as workers and
 * device memory free up (vfgpu_memory_estimate against the server's budget).  Each
 * admitted problem runs on a ctx of its grid size taken from a pool: contexts
 * (fields, solver work space, captured CUDA graphs) are kept after a problem ends
 * and reused by the next problem of the same size; idle contexts of other sizes
 * are evicted when memory is short.  Problems on different workers overlap on the
 * device through their own streams.  The kernels are deterministic, so a problem
 * gives the same bits alone and in any mix. */
#define VFGPU_SERVE_MAX_PENNY 16
#define VFGPU_SERVE_MAX_RECT 16
typedef struct {
  vfgpu_grid grid;
  vfgpu_matprop mp;            /* one layer */
  vfgpu_vfprop vf;
  vfgpu_bc bcU[3], bcV;
  double pressure;             /* uniform crack pressure (used when vf.hasCrackPressure) */
  int npenny, nrect;
  vfgpu_penny penny[VFGPU_SERVE_MAX_PENNY];
  vfgpu_rect rect[VFGPU_SERVE_MAX_RECT];
  int am_its;                  /* AM iterations: exactly am_its if > 0 ...              */
  double altmintol;            /* ... else until ||V - Vold||_inf < altmintol           */
  int max_am_its;              /*     or max_am_its iterations                          */
  vfgpu_solve_opts opts;       /* precision and tolerances of both solves               */
  double* out_u;               /* optional host buffers filled at the end: 3N, N, N     */
  double* out_v;
  double* out_cellcov;         /* optional ((nx-1)(ny-1)(nz-1)) */
  unsigned long long tag;      /* caller's id, returned in the result */
} vfgpu_request;

typedef struct {
  unsigned long long ticket, tag;
  int status;                  /* VFGPU_OK, or the first failing call's code            */
  int am_its, ksp_its_u, ksp_its_v;
  double am_err;               /* last ||V - Vold||_inf */
  double elastic, pressure_work, surface, cov;
  double t_submit, t_start, t_done;  /* seconds on the server clock */
  int worker;
  int reused_ctx;              /* 1 if the problem ran on a pooled ctx */
  char error[160];             /* message of the failing call, "" if status == VFGPU_OK */
} vfgpu_result;

typedef struct {
  long long budget_bytes, reserved_bytes, peak_reserved_bytes;
  int workers, contexts, contexts_created, evictions;
  long long submitted, completed, queued, running;
} vfgpu_server_info;

typedef struct vfgpu_server vfgpu_server;
/* workers >= 1 threads on CUDA device `device`; budget_bytes <= 0 means 85% of the
 * device memory free at creation. */
int vfgpu_server_create(int device, int workers, long long budget_bytes, vfgpu_server** out);
/* Copies the request and queues it; *ticket identifies its result.  Never blocks. */
int vfgpu_server_submit(vfgpu_server* s, const vfgpu_request* req, unsigned long long* ticket);
/* Waits up to timeout_s (< 0: for ever) for the next finished problem, in completion
 * order.  Returns VFGPU_OK with *res filled, or VFGPU_NOT_CONVERGED on timeout. */
int vfgpu_server_next(vfgpu_server* s, double timeout_s, vfgpu_result* res);
/* Seconds since the server was created (the clock of the result time stamps). */
double vfgpu_server_clock(vfgpu_server* s);
int vfgpu_server_info_get(vfgpu_server* s, vfgpu_server_info* info);
/* Finishes the queued and running problems, joins the workers, frees every ctx. */
int vfgpu_server_destroy(vfgpu_server* s);

/* No counterpart in the reference.  y = K(v) x like vfgpu_u_apply (FP64, one
 * homogeneous material, Dirichlet rows from bcbits), for callers that cannot
 * allocate device memory while they run -- e.g. a matrix-shell callback inside
 * an external solver whose host program owns every device buffer, or a loop
 * that cannot afford cudaMalloc's device-wide synchronisation.  No ctx is
 * needed and nothing is allocated: v (N), x and y (3N) and bcbits (N bytes,
 * bit c set = component c of the node is Dirichlet; may be NULL) are device
 * arrays of the current device, the work is queued on `stream` (a
 * cudaStream_t, NULL = legacy default stream) and the call returns without
 * waiting.  The only scratch (the seam partial sums) is a fixed 32 MiB array
 * inside the library (VFGPU_NOALLOC_SCRATCH_DOUBLES doubles; every GPU that
 * loads the library holds it until exit); grids whose seams need more are
 * rejected with VFGPU_ERR_INVALID (129^3 fits, 161^3 does not), and so are x and y
 * that overlap (the apply is out of place).  Every call looks up the array's device
 * address in the current context (cudaGetSymbolAddress, host-side) and, on the first
 * call on a device, opts the kernels in to their shared memory: make that first call
 * before any stream capture.  All calls share the one array, so calls whose work
 * overlaps on the GPU (different streams, different threads) race; serialise them.
 * Every scratch slot read is written earlier in the same call, so no clearing is
 * needed between calls. */
#define VFGPU_NOALLOC_SCRATCH_DOUBLES 4194304
int vfgpu_u_apply_noalloc(const vfgpu_grid* grid, const vfgpu_matprop* mp, double eta,
                          const double* v, const unsigned char* bcbits, const double* x,
                          double* y, void* stream);

/* No counterpart in the reference: y = J_U x (FP32 vectors on the device, V from the
 * ctx) with the element contraction on the tensor cores -- two GEMMs per tile of 128
 * elements (gradients, strains and v at the 27 Gauss points from the 32 nodal values;
 * the Gauss-weighted transpose back to the 24 nodal forces) issued as tcgen05.mma in
 * split TF32 (hi/lo, three products per term, FP32 accumulation in tensor memory), the
 * pointwise degradation v^2 + eta and Lame factors on the CUDA cores.  Element results
 * are summed with atomics (not bit-reproducible); Dirichlet rows y = x.  A measured
 * alternative to vfgpu_u_apply_dev's CUDA-core element, not used by the solvers;
 * UNILATERAL_NONE only.  Queued on the ctx stream; vfgpu_tc_error (synchronous) reports
 * whether a bounded wait inside the last call gave up (its results are then void). */
int vfgpu_u_apply_tc(vfgpu_ctx* ctx, const float* x, float* y);
int vfgpu_tc_error(vfgpu_ctx* ctx, int* flagged);
/* Host only: the two constant matrices of vfgpu_u_apply_tc for an hx x hy x hz cell,
 * row-major B1[32][224] (K = 24 displacements + 8 phase-field values, N = 27 points x
 * {tr, 2 e_xx, 2 e_yy, 2 e_zz, g_xy, g_xz, g_yz, v} + 8 zero columns) and B2[192][32]
 * (K = 3 passes x (9 points x {lambda s tr, mu s E_xx .. E_yz} + 1 zero row), N = 24
 * dofs + 8 zero columns). */
int vfgpu_tc_tables(double hx, double hy, double hz, double* B1, double* B2);

/* Measurement utility, no counterpart in the reference: FMA throughput of the
 * current GPU's CUDA cores in TFLOP/s for bytes = 8 (FP64) or 4 (FP32), from a
 * kernel of independent FMA chains (the denominator of the operator's compute
 * roofline). */
int vfgpu_fma_peak(int bytes, double* tflops);

/* Diagnostic, no counterpart in the reference: runs the bounded mbarrier wait that the
 * V apply's coefficient copies use on a phase that completes (complete = 1) or never
 * does (complete = 0) with a limit of `cycles` (<= 4e9) SM clock cycles, and sets
 * *timed_out to whether the wait gave up (the kernel then returns normally and the
 * device stays usable).  Returns 0, or < 0 on a bad argument or CUDA error. */
int vfgpu_wait_selftest(long long cycles, int complete, int* timed_out);

#ifdef __cplusplus
}
#endif
#endif /* VFGPU_H */
