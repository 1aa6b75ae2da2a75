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
#include <stdlib.h>
#include <string.h>

typedef void (*apply_fn)(void *ctx, const double *x, double *y);

static double dot(int64_t n, const double *a, const double *b) {
  double s = 0.;
  for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* KSPSolve_CG with KSP_NORM_PRECONDITIONED and KSPConvergedDefault:
 * converged when ||z|| <= max(rtol ||z0||, atol); x0 = 0 (SNES linear solves).
 * Rows with active[i] != 0 are excluded (reduced-space solves): they keep x=0. */
static int pcg(int64_t n, apply_fn A, void *ctx, const double *dinv, const double *b,
               double *x, const uint8_t *active, const vfo_solver_opts *o, int *its_out) {
  double *r = malloc(n * sizeof(double)), *z = malloc(n * sizeof(double));
  double *p = malloc(n * sizeof(double)), *w = malloc(n * sizeof(double));
  for (int64_t i = 0; i < n; i++) {
    x[i] = 0.;
    r[i] = (active && active[i]) ? 0. : b[i];
    z[i] = r[i] * dinv[i];
  }
  double dp = sqrt(dot(n, z, z)), rnorm0 = dp, ttol = fmax(o->rtol * rnorm0, o->atol);
  int its = 0, reason = 0;
  if (dp <= ttol) reason = 1;
  double beta = dot(n, z, r), betaold = 0.;
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
    double dpi = dot(n, p, w);
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
    dp = sqrt(dot(n, z, z));
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
    beta = dot(n, z, r);
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
    int kr = pcg(n, u_apply_cb, &c, dinv, F, Y, NULL, o, &kits);
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
    int kr = pcg(n, v_apply_cb, &c, dinv, F, Y, act, o, &kits);
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
