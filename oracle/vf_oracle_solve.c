/*
 * vf_oracle_solve.c -- PETSc solver semantics restated for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference configures (VFCommon.c:1005-1088):
 *   snesU: SNESNEWTONLS, L2 line search, atol = rtol = 1e-8; KSPCG rtol 1e-8,
 *          atol 1e-10, PC jacobi (the configs' -U_pc_type jacobi);
 *   snesV: SNESVINEWTONRSLS, bounds [0,1] (AT1: [0,VIrrev], VFCommon.c:1149-1154),
 *          atol = rtol = 1e-8; KSPCG + Jacobi on the inactive set.
 * PETSc is an external dependency (version unpinned beyond ">= 3.10",
 * README.md:29) that is absent here; these routines restate the published
 * algorithms: preconditioned CG with the default convergence test on the
 * preconditioned residual norm, Newton with a quadratic-fit (L2) line search,
 * and the reduced-space active-set VI Newton method.
 */
#include "vf_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef void (*apply_fn)(void *ctx, const double *x, double *y);

static double dot(int64_t n, const double *a, const double *b) {
  double s = 0.;
  for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* The same sum spread over the threads (the assembled-method baseline: PETSc's
 * VecDot runs on every rank). */
static double pdot(int64_t n, const double *a, const double *b) {
  double s = 0.;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* KSPSolve_CG with KSP_NORM_PRECONDITIONED and KSPConvergedDefault:
 * converged when ||z|| <= max(rtol ||z0||, atol); x0 = 0 (SNES linear solves).
 * Rows with active[i] != 0 are excluded (reduced-space solves): they keep x=0. */
static int pcg(int64_t n, apply_fn A, void *ctx, const double *dinv, const double *b,
               double *x, const uint8_t *active, const vfo_solver_opts *o, int *its_out,
               int par) {
  double (*dotf)(int64_t, const double *, const double *) = par ? pdot : dot;
  double *r = malloc(n * sizeof(double)), *z = malloc(n * sizeof(double));
  double *p = malloc(n * sizeof(double)), *w = malloc(n * sizeof(double));
  for (int64_t i = 0; i < n; i++) {
    x[i] = 0.;
    r[i] = (active && active[i]) ? 0. : b[i];
    z[i] = r[i] * dinv[i];
  }
  double dp = sqrt(dotf(n, z, z)), rnorm0 = dp, ttol = fmax(o->rtol * rnorm0, o->atol);
  int its = 0, reason = 0;
  if (dp <= ttol) reason = 1;
  double beta = dotf(n, z, r), betaold = 0.;
  while (!reason && its < o->maxit) {
    if (beta == 0.) {
      reason = 1;
      break;
    }
    if (its == 0)
      memcpy(p, z, n * sizeof(double));
    else {
      double bb = beta / betaold;
      for (int64_t i = 0; i < n; i++) p[i] = z[i] + bb * p[i];
    }
    A(ctx, p, w);
    if (active)
      for (int64_t i = 0; i < n; i++)
        if (active[i]) w[i] = 0.;
    double dpi = dotf(n, p, w);
    if (!(dpi > 0.)) {
      reason = -8; /* KSP_DIVERGED_INDEFINITE_MAT */
      break;
    }
    double a = beta / dpi;
    for (int64_t i = 0; i < n; i++) {
      x[i] += a * p[i];
      r[i] -= a * w[i];
      z[i] = r[i] * dinv[i];
    }
    dp = sqrt(dotf(n, z, z));
    its++;
    if (dp <= ttol) {
      reason = 1;
      break;
    }
    if (dp != dp || dp >= o->dtol * rnorm0) {
      reason = -4;
      break;
    }
    betaold = beta;
    beta = dotf(n, z, r);
  }
  free(r);
  free(z);
  free(p);
  free(w);
  *its_out = its;
  return reason;
}

/* ------------------------------------------------------------------------ */
typedef struct {
  const vfo_problem *P;
  const double *u0, *v;
  const uint8_t *bcmask;
} uctx;

static void u_apply_cb(void *c, const double *x, double *y) {
  uctx *u = (uctx *)c;
  vfo_u_apply_mf_u(u->P, u->u0, u->v, x, u->bcmask, y);
}

typedef struct {
  const vfo_problem *P;
  const double *v, *theta, *thetaRef, *p;
  double *f;  /* work space for the load */
} uload;

/* F(u) = K(v; u) u - f(u), BC rows u - ubc (VF_UResidual semantics); the load and,
 * for NOCOMPRESSION, the operator depend on u through the sign of tr(eps(u)). */
static void u_func(const uload *L, const uint8_t *bc, const double *bcval, const double *u,
                   double *F) {
  const vfo_problem *P = L->P;
  int64_t n = 3 * (int64_t)P->nx * P->ny * P->nz;
  vfo_u_rhs_u(P, u, L->v, L->theta, L->thetaRef, L->p, L->f);
  vfo_u_apply_mf_u(P, u, L->v, u, NULL, F);
  for (int64_t i = 0; i < n; i++) F[i] = bc[i] ? u[i] - bcval[i] : F[i] - L->f[i];
}

/* VF_StepU = SNESSolve(snesU): SNESNEWTONLS + SNESLINESEARCHL2 (one secant step on
 * the derivative of ||F(x - lambda Y)||^2 fitted from lambda = 0, 1/2, 1).  For the
 * affine U residual that lands on the exact minimiser; for NOCOMPRESSION the
 * residual is piecewise affine, the Jacobian K(v; u) is re-formed at every Newton
 * iterate (VF_UIJacobian, VFMech.c:1942-1980) and so are the Jacobi diagonal and
 * the load. */
int vfo_step_u(const vfo_problem *P, double *u, const double *v, const double *theta,
               const double *thetaRef, const double *p, const uint8_t *bcmask,
               const double *bcval, const vfo_solver_opts *o, vfo_stats *st) {
  int64_t n = 3 * (int64_t)P->nx * P->ny * P->nz;
  double *f = malloc(n * sizeof(double)), *F = malloc(n * sizeof(double));
  double *Y = malloc(n * sizeof(double)), *W = malloc(n * sizeof(double));
  double *Fw = malloc(n * sizeof(double)), *dinv = malloc(n * sizeof(double));
  uload L = {P, v, theta, thetaRef, p, f};
  vfo_u_diag_u(P, u, v, bcmask, dinv);
  for (int64_t i = 0; i < n; i++) dinv[i] = 1. / dinv[i];
  u_func(&L, bcmask, bcval, u, F);
  double fnorm = sqrt(dot(n, F, F));
  memset(st, 0, sizeof *st);
  st->fnorm0 = fnorm;
  double ttol = o->snes_rtol * fnorm;
  int reason = 0;
  if (fnorm < o->snes_atol) reason = 2;
  double *u0 = malloc(n * sizeof(double));
  uctx c = {P, u0, v, bcmask};
  for (int it = 0; !reason && it < o->snes_maxit; it++) {
    int kits = 0;
    memcpy(u0, u, n * sizeof(double));  /* the Jacobian's linearisation point */
    if (P->unilateral && it > 0) {
      vfo_u_diag_u(P, u, v, bcmask, dinv);
      for (int64_t i = 0; i < n; i++) dinv[i] = 1. / dinv[i];
    }
    int kr = pcg(n, u_apply_cb, &c, dinv, F, Y, NULL, o, &kits, 0);
    st->ksp_its += kits;
    if (kr < 0) {
      reason = -3; /* SNES_DIVERGED_LINEAR_SOLVE */
      break;
    }
    /* L2 line search: samples at lambda = 0, 1/2, 1. */
    double q0 = fnorm * fnorm, qm, q1;
    for (int64_t i = 0; i < n; i++) W[i] = u[i] - 0.5 * Y[i];
    u_func(&L, bcmask, bcval, W, Fw);
    qm = dot(n, Fw, Fw);
    for (int64_t i = 0; i < n; i++) W[i] = u[i] - Y[i];
    u_func(&L, bcmask, bcval, W, Fw);
    q1 = dot(n, Fw, Fw);
    double dE = 3. * q1 - 4. * qm + q0, dE_old = -3. * q0 + 4. * qm - q1;
    double lambda = 1.;
    if (dE - dE_old != 0.) {
      double lu = 1. - dE / (dE - dE_old);
      if (lu == lu && lu > 1e-12) lambda = lu;
    }
    for (int64_t i = 0; i < n; i++) u[i] -= lambda * Y[i];
    u_func(&L, bcmask, bcval, u, F);
    fnorm = sqrt(dot(n, F, F));
    double ynorm = lambda * sqrt(dot(n, Y, Y)), xnorm = sqrt(dot(n, u, u));
    st->newton_its = it + 1;
    if (fnorm != fnorm)
      reason = -4;
    else if (fnorm < o->snes_atol)
      reason = 2;
    else if (fnorm <= ttol)
      reason = 3;
    else if (ynorm < o->snes_stol * xnorm)
      reason = 4;
  }
  if (!reason) reason = -5; /* SNES_DIVERGED_MAX_IT */
  st->reason = reason;
  st->fnorm = fnorm;
  free(f);
  free(F);
  free(Y);
  free(W);
  free(Fw);
  free(dinv);
  free(u0);
  return 0;
}

/* ------------------------------------------------------------------------ */
typedef struct {
  const vfo_problem *P;
  const double *u, *theta, *thetaRef, *virrev;
  const uint8_t *bcmask;
} vctx;

static void v_apply_cb(void *c, const double *x, double *y) {
  vctx *q = (vctx *)c;
  vfo_v_apply(q->P, q->u, q->theta, q->thetaRef, q->virrev, q->bcmask, x, y);
}

/* SNESVIComputeInactiveSetFnorm semantics. */
static double vi_fnorm(int64_t n, const double *F, const double *x, const double *lb,
                       const double *ub) {
  double s = 0.;
  for (int64_t i = 0; i < n; i++)
    if ((x[i] > lb[i] + 1.e-8 || F[i] <= 0.) && (x[i] < ub[i] - 1.e-8 || F[i] >= 0.))
      s += F[i] * F[i];
  return sqrt(s);
}

static void v_func(const vfo_problem *P, vctx *c, const double *b, const double *bcval,
                   const double *v, double *F) {
  int64_t n = (int64_t)P->nx * P->ny * P->nz;
  vfo_v_apply(P, c->u, c->theta, c->thetaRef, NULL, NULL, v, F);
  for (int64_t i = 0; i < n; i++) {
    F[i] -= b[i];
    if (P->atnum == 2 && c->virrev && c->virrev[i] <= P->irrevtol) F[i] = 0.;
    if (c->bcmask && c->bcmask[i]) F[i] = v[i] - bcval[i];
  }
}

/* VF_StepV = SNESSolve(snesV) with SNESVINEWTONRSLS: active set
 * A = {x <= l+1e-8 and F >= 0} U {x >= u-1e-8 and F <= 0}, Newton step on the
 * inactive set, projected back-tracking line search (BT, alpha = 0). */
int vfo_step_v(const vfo_problem *P, double *v, const double *u, const double *theta,
               const double *thetaRef, const double *p, const double *virrev,
               const double *lb, const double *ub, const uint8_t *bcmask,
               const double *bcval, const vfo_solver_opts *o, vfo_stats *st) {
  int64_t n = (int64_t)P->nx * P->ny * P->nz;
  double *b = malloc(n * sizeof(double)), *F = malloc(n * sizeof(double));
  double *Y = malloc(n * sizeof(double)), *W = malloc(n * sizeof(double));
  double *Fw = malloc(n * sizeof(double)), *dinv = malloc(n * sizeof(double));
  uint8_t *act = malloc(n);
  vctx c = {P, u, theta, thetaRef, virrev, bcmask};
  vfo_v_rhs(P, u, p, b);
  vfo_v_diag(P, u, theta, thetaRef, virrev, bcmask, dinv);
  for (int64_t i = 0; i < n; i++) dinv[i] = 1. / dinv[i];
  for (int64_t i = 0; i < n; i++) v[i] = fmin(fmax(v[i], lb[i]), ub[i]);
  v_func(P, &c, b, bcval, v, F);
  double fnorm = vi_fnorm(n, F, v, lb, ub);
  memset(st, 0, sizeof *st);
  st->fnorm0 = fnorm;
  double ttol = o->snes_rtol * fnorm;
  int reason = 0;
  if (fnorm < o->snes_atol) reason = 2;
  for (int it = 0; !reason && it < o->snes_maxit; it++) {
    for (int64_t i = 0; i < n; i++)
      act[i] = !((v[i] > lb[i] + 1.e-8 || F[i] < 0.) && (v[i] < ub[i] - 1.e-8 || F[i] > 0.));
    int kits = 0;
    int kr = pcg(n, v_apply_cb, &c, dinv, F, Y, act, o, &kits, 0);
    st->ksp_its += kits;
    if (kr < 0) {
      reason = -3;
      break;
    }
    double lambda = 1., gnorm = 0.;
    for (int bt = 0; bt < 30; bt++) {
      for (int64_t i = 0; i < n; i++) W[i] = fmin(fmax(v[i] - lambda * Y[i], lb[i]), ub[i]);
      v_func(P, &c, b, bcval, W, Fw);
      gnorm = vi_fnorm(n, Fw, W, lb, ub);
      if (gnorm <= fnorm || lambda < 1e-12) break;
      lambda *= 0.5;
    }
    double ynorm = 0.;
    for (int64_t i = 0; i < n; i++) {
      ynorm += (W[i] - v[i]) * (W[i] - v[i]);
      v[i] = W[i];
      F[i] = Fw[i];
    }
    ynorm = sqrt(ynorm);
    fnorm = gnorm;
    double xnorm = sqrt(dot(n, v, v));
    st->newton_its = it + 1;
    if (fnorm != fnorm)
      reason = -4;
    else if (fnorm < o->snes_atol)
      reason = 2;
    else if (fnorm <= ttol)
      reason = 3;
    else if (ynorm < o->snes_stol * xnorm)
      reason = 4;
  }
  if (!reason) reason = -5;
  st->reason = reason;
  st->fnorm = fnorm;
  free(b);
  free(F);
  free(Y);
  free(W);
  free(Fw);
  free(dinv);
  free(act);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* The reference's method on the host cores: the CPU AM-step baseline.
 * VF_StepU / VF_StepV as VPFHF runs them: every residual evaluation re-forms the
 * element matrices (VF_UResidual, VFMech.c:1555-1596; VF_VResidual, VFMech.c:2772-2848),
 * every Newton iteration assembles the Jacobian into an AIJ (CSR) matrix
 * (VF_UIJacobian, VFMech.c:1897-2029; VF_VIJacobian, VFMech.c:2948-3027), and KSPCG +
 * Jacobi runs on the assembled matrix, one SpMV per iteration.  Same Newton / line
 * search / VI logic and stopping tests as vfo_step_u / vfo_step_v; the element loops
 * run in 8 parity colours on all threads (the reference spreads them over MPI ranks).
 * UNILATERAL_NONE only.  Used to time the CPU baseline; the tests check its solutions
 * against vfo_step_u / vfo_step_v. */

#define ONODE(P, i, j, k) (((int64_t)(k) * (P)->ny + (j)) * (P)->nx + (i))

typedef struct {
  int64_t n;
  int64_t *rowptr;
  int32_t *col;
  double *val;
  int nthreads;
} csr_t;

static void csr_apply_cb(void *c, const double *x, double *y) {
  csr_t *A = (csr_t *)c;
  vfo_csr_spmv(A->n, A->rowptr, A->col, A->val, x, y, A->nthreads);
}

static void csr_free(csr_t *A) {
  free(A->rowptr);
  free(A->col);
  free(A->val);
}

static void csr_dinv(const csr_t *A, double *dinv) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < A->n; r++) {
    double d = 0.;
    for (int64_t q = A->rowptr[r]; q < A->rowptr[r + 1]; q++)
      if (A->col[q] == r) d = A->val[q];
    dinv[r] = 1. / d;
  }
}

static void cell_nodes8(const vfo_problem *P, int ei, int ej, int ek, int64_t n[8]) {
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) n[i + 2 * j + 4 * k] = ONODE(P, ei + i, ej + j, ek + k);
}

/* The colour classes of the element loop: colour c holds the cells whose index parities
 * are (c & 1, c >> 1 & 1, c >> 2 & 1); no two cells of a class share a node. */
#define COLOURED_CELLS(P, ei, ej, ek, BODY)                                                \
  for (int color = 0; color < 8; color++) {                                                \
    int cx_ = color & 1, cy_ = (color >> 1) & 1, cz_ = (color >> 2) & 1;                   \
    int hx_ = ((P)->nx - 1 - cx_ + 1) / 2, hy_ = ((P)->ny - 1 - cy_ + 1) / 2;              \
    int hz_ = ((P)->nz - 1 - cz_ + 1) / 2;                                                 \
    int64_t tot_ = (int64_t)hx_ * hy_ * hz_;                                               \
    _Pragma("omp parallel for schedule(static)") for (int64_t t_ = 0; t_ < tot_; t_++) {   \
      int ei = cx_ + 2 * (int)(t_ % hx_);                                                  \
      int ej = cy_ + 2 * (int)((t_ / hx_) % hy_);                                          \
      int ek = cz_ + 2 * (int)(t_ / ((int64_t)hx_ * hy_));                                 \
      BODY                                                                                 \
    }                                                                                      \
  }

/* F = K(v) u - f by element matrices, BC rows u - bcval. */
static void u_res_elem(const vfo_problem *P, const double *u, const double *v, const double *f,
                       const uint8_t *bc, const double *bcval, double *F) {
  int64_t n3 = 3 * (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < n3; q++) F[q] = -f[q];
  COLOURED_CELLS(P, ei, ej, ek, {
    double K[576];
    int64_t n[8];
    vfo_u_element_matrix(P, ei, ej, ek, v, K);
    cell_nodes8(P, ei, ej, ek, n);
    for (int a = 0, l = 0; a < 8; a++)
      for (int c1 = 0; c1 < 3; c1++) {
        double s = 0.;
        for (int b = 0; b < 8; b++)
          for (int c2 = 0; c2 < 3; c2++, l++) s += K[l] * u[3 * n[b] + c2];
        F[3 * n[a] + c1] += s;
      }
  })
  if (bc)
    for (int64_t q = 0; q < n3; q++)
      if (bc[q]) F[q] = u[q] - bcval[q];
}

int vfo_step_u_asm(const vfo_problem *P, double *u, const double *v, const double *theta,
                   const double *thetaRef, const double *p, const uint8_t *bcmask,
                   const double *bcval, const vfo_solver_opts *o, vfo_stats *st,
                   double *seconds_assembly) {
  int64_t n = 3 * (int64_t)P->nx * P->ny * P->nz;
  double *f = malloc(n * sizeof(double)), *F = malloc(n * sizeof(double));
  double *Y = malloc(n * sizeof(double)), *W = malloc(n * sizeof(double));
  double *Fw = malloc(n * sizeof(double)), *dinv = malloc(n * sizeof(double));
  csr_t A = {n, malloc((n + 1) * sizeof(int64_t)), NULL, NULL, P->nthreads};
  int64_t nnz = vfo_u_csr_nnz(P);
  A.col = malloc(nnz * sizeof(int32_t));
  A.val = malloc(nnz * sizeof(double));
  double tasm = 0.;
  vfo_u_rhs(P, v, theta, thetaRef, p, f);
  u_res_elem(P, u, v, f, bcmask, bcval, F);
  double fnorm = sqrt(pdot(n, F, F));
  memset(st, 0, sizeof *st);
  st->fnorm0 = fnorm;
  double ttol = o->snes_rtol * fnorm;
  int reason = 0;
  if (fnorm < o->snes_atol) reason = 2;
  for (int it = 0; !reason && it < o->snes_maxit; it++) {
    double t0 = omp_get_wtime();
    vfo_u_assemble_csr(P, v, bcmask, A.rowptr, A.col, A.val);
    csr_dinv(&A, dinv);
    tasm += omp_get_wtime() - t0;
    int kits = 0;
    int kr = pcg(n, csr_apply_cb, &A, dinv, F, Y, NULL, o, &kits, 1);
    st->ksp_its += kits;
    if (kr < 0) {
      reason = -3;
      break;
    }
    double q0 = fnorm * fnorm, qm, q1;
    for (int64_t i = 0; i < n; i++) W[i] = u[i] - 0.5 * Y[i];
    u_res_elem(P, W, v, f, bcmask, bcval, Fw);
    qm = pdot(n, Fw, Fw);
    for (int64_t i = 0; i < n; i++) W[i] = u[i] - Y[i];
    u_res_elem(P, W, v, f, bcmask, bcval, Fw);
    q1 = pdot(n, Fw, Fw);
    double dE = 3. * q1 - 4. * qm + q0, dE_old = -3. * q0 + 4. * qm - q1;
    double lambda = 1.;
    if (dE - dE_old != 0.) {
      double lu = 1. - dE / (dE - dE_old);
      if (lu == lu && lu > 1e-12) lambda = lu;
    }
    for (int64_t i = 0; i < n; i++) u[i] -= lambda * Y[i];
    u_res_elem(P, u, v, f, bcmask, bcval, F);
    fnorm = sqrt(pdot(n, F, F));
    double ynorm = lambda * sqrt(pdot(n, Y, Y)), xnorm = sqrt(pdot(n, u, u));
    st->newton_its = it + 1;
    if (fnorm != fnorm)
      reason = -4;
    else if (fnorm < o->snes_atol)
      reason = 2;
    else if (fnorm <= ttol)
      reason = 3;
    else if (ynorm < o->snes_stol * xnorm)
      reason = 4;
  }
  if (!reason) reason = -5;
  st->reason = reason;
  st->fnorm = fnorm;
  if (seconds_assembly) *seconds_assembly = tasm;
  csr_free(&A);
  free(f);
  free(F);
  free(Y);
  free(W);
  free(Fw);
  free(dinv);
  return 0;
}

/* The V Jacobian (27-point box stencil, columns ascending) with the fixed dofs
 * (Dirichlet, AT2 irreversibility) made identity rows and columns
 * (MatApplyDirichletBCRowCol, VFCartFE.c:1305-1454; VF_IrrevApplyEQMat,
 * VFMech.c:2637-2682). */
static void v_assemble_csr(const vfo_problem *P, const double *u, const double *theta,
                           const double *thetaRef, const uint8_t *fixed, csr_t *A) {
  int64_t r = 0;
  A->rowptr[0] = 0;
  for (int k = 0; k < P->nz; k++)
    for (int j = 0; j < P->ny; j++)
      for (int i = 0; i < P->nx; i++, r++) {
        int64_t pos = A->rowptr[r];
        for (int kk = k - 1; kk <= k + 1; kk++)
          for (int jj = j - 1; jj <= j + 1; jj++)
            for (int ii = i - 1; ii <= i + 1; ii++) {
              if (ii < 0 || jj < 0 || kk < 0 || ii >= P->nx || jj >= P->ny || kk >= P->nz) continue;
              A->col[pos] = (int32_t)ONODE(P, ii, jj, kk);
              A->val[pos] = 0.;
              pos++;
            }
        A->rowptr[r + 1] = pos;
      }
  COLOURED_CELLS(P, ei, ej, ek, {
    double K[64];
    int64_t n[8];
    vfo_v_element_matrix(P, ei, ej, ek, u, theta, thetaRef, K);
    cell_nodes8(P, ei, ej, ek, n);
    for (int a = 0; a < 8; a++)
      for (int b = 0; b < 8; b++) {
        int64_t q = A->rowptr[n[a]];
        while (A->col[q] != n[b]) q++;
        A->val[q] += K[a * 8 + b];
      }
  })
#pragma omp parallel for schedule(static)
  for (int64_t row = 0; row < A->n; row++)
    for (int64_t q = A->rowptr[row]; q < A->rowptr[row + 1]; q++) {
      const int64_t c = A->col[q];
      if (fixed[row] || fixed[c]) A->val[q] = (c == row) ? 1. : 0.;
    }
}

/* F_V = K_V(u) v - b by element matrices; AT2 irreversibility rows 0; BC rows v - bc. */
static void v_res_elem(const vfo_problem *P, const double *u, const double *theta,
                       const double *thetaRef, const double *b, const double *virrev,
                       const uint8_t *bcmask, const double *bcval, const double *v, double *F) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < N; q++) F[q] = -b[q];
  COLOURED_CELLS(P, ei, ej, ek, {
    double K[64];
    int64_t n[8];
    vfo_v_element_matrix(P, ei, ej, ek, u, theta, thetaRef, K);
    cell_nodes8(P, ei, ej, ek, n);
    for (int a = 0; a < 8; a++) {
      double s = 0.;
      for (int c = 0; c < 8; c++) s += K[a * 8 + c] * v[n[c]];
      F[n[a]] += s;
    }
  })
  for (int64_t q = 0; q < N; q++) {
    if (P->atnum == 2 && virrev && virrev[q] <= P->irrevtol) F[q] = 0.;
    if (bcmask && bcmask[q]) F[q] = v[q] - bcval[q];
  }
}

int vfo_step_v_asm(const vfo_problem *P, double *v, const double *u, const double *theta,
                   const double *thetaRef, const double *p, const double *virrev,
                   const double *lb, const double *ub, const uint8_t *bcmask,
                   const double *bcval, const vfo_solver_opts *o, vfo_stats *st,
                   double *seconds_assembly) {
  int64_t n = (int64_t)P->nx * P->ny * P->nz;
  double *b = malloc(n * sizeof(double)), *F = malloc(n * sizeof(double));
  double *Y = malloc(n * sizeof(double)), *W = malloc(n * sizeof(double));
  double *Fw = malloc(n * sizeof(double)), *dinv = malloc(n * sizeof(double));
  uint8_t *act = malloc(n), *fixed = malloc(n);
  for (int64_t q = 0; q < n; q++)
    fixed[q] = (bcmask && bcmask[q]) || (P->atnum == 2 && virrev && virrev[q] <= P->irrevtol);
  csr_t A = {n, malloc((n + 1) * sizeof(int64_t)), NULL, NULL, P->nthreads};
  A.col = malloc(27 * n * sizeof(int32_t));
  A.val = malloc(27 * n * sizeof(double));
  vfo_v_rhs(P, u, p, b);
  double tasm = 0.;
  for (int64_t i = 0; i < n; i++) v[i] = fmin(fmax(v[i], lb[i]), ub[i]);
  v_res_elem(P, u, theta, thetaRef, b, virrev, bcmask, bcval, v, F);
  double fnorm = vi_fnorm(n, F, v, lb, ub);
  memset(st, 0, sizeof *st);
  st->fnorm0 = fnorm;
  double ttol = o->snes_rtol * fnorm;
  int reason = 0;
  if (fnorm < o->snes_atol) reason = 2;
  for (int it = 0; !reason && it < o->snes_maxit; it++) {
    /* the V Jacobian does not depend on v, but VINEWTONRSLS calls VF_VIJacobian at
     * every Newton iteration, which assembles it again */
    double t0 = omp_get_wtime();
    v_assemble_csr(P, u, theta, thetaRef, fixed, &A);
    csr_dinv(&A, dinv);
    tasm += omp_get_wtime() - t0;
    for (int64_t i = 0; i < n; i++)
      act[i] = !((v[i] > lb[i] + 1.e-8 || F[i] < 0.) && (v[i] < ub[i] - 1.e-8 || F[i] > 0.));
    int kits = 0;
    int kr = pcg(n, csr_apply_cb, &A, dinv, F, Y, act, o, &kits, 1);
    st->ksp_its += kits;
    if (kr < 0) {
      reason = -3;
      break;
    }
    double lambda = 1., gnorm = 0.;
    for (int bt = 0; bt < 30; bt++) {
      for (int64_t i = 0; i < n; i++) W[i] = fmin(fmax(v[i] - lambda * Y[i], lb[i]), ub[i]);
      v_res_elem(P, u, theta, thetaRef, b, virrev, bcmask, bcval, W, Fw);
      gnorm = vi_fnorm(n, Fw, W, lb, ub);
      if (gnorm <= fnorm || lambda < 1e-12) break;
      lambda *= 0.5;
    }
    double ynorm = 0.;
    for (int64_t i = 0; i < n; i++) {
      ynorm += (W[i] - v[i]) * (W[i] - v[i]);
      v[i] = W[i];
      F[i] = Fw[i];
    }
    ynorm = sqrt(ynorm);
    fnorm = gnorm;
    double xnorm = sqrt(pdot(n, v, v));
    st->newton_its = it + 1;
    if (fnorm != fnorm)
      reason = -4;
    else if (fnorm < o->snes_atol)
      reason = 2;
    else if (fnorm <= ttol)
      reason = 3;
    else if (ynorm < o->snes_stol * xnorm)
      reason = 4;
  }
  if (!reason) reason = -5;
  st->reason = reason;
  st->fnorm = fnorm;
  if (seconds_assembly) *seconds_assembly = tasm;
  csr_free(&A);
  free(b);
  free(F);
  free(Y);
  free(W);
  free(Fw);
  free(dinv);
  free(act);
  free(fixed);
  return 0;
}
