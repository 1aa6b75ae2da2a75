/*
 * vf_oracle.c -- FP64 CPU restatement of the VPFHF hot-path arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline; never
 * linked into the product).  Every "_ref" function follows the reference's
 * loop nesting and left-to-right expression order so that it reproduces the
 * reference's FP64 rounding on a single rank; the "_mf" / fast variants are
 * algebraically identical reorderings used where speed matters.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include "vf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NODE(P, i, j, k) (((int64_t)(k) * (P)->ny + (j)) * (P)->nx + (i))

/* ------------------------------------------------------------------------ */
/* Geometry: VFGeometryInitialize builds X[i] = i*lx/(nx-1.) (VFCommon.c:394-399)
 * and every element loop takes hx = X[ei+1]-X[ei] (e.g. VFMech.c:1557-1559). */
static double coord(int i, double l, int n) { return i == 0 ? 0. : i * l / (n - 1.); }

static void cell_h(const vfo_problem *P, int ei, int ej, int ek, double *hx, double *hy,
                   double *hz) {
  *hx = coord(ei + 1, P->lx, P->nx) - coord(ei, P->lx, P->nx);
  *hy = coord(ej + 1, P->ly, P->ny) - coord(ej, P->ly, P->ny);
  *hz = coord(ek + 1, P->lz, P->nz) - coord(ek, P->lz, P->nz);
}

typedef struct {
  double lambda, mu, alpha, beta, Gc;
} cellmat;

/* Lame coefficients as VFMatPropGet computes them (VFCommon.c:583-586); the
 * optional per-cell E is this build's generalisation of the per-layer table. */
static cellmat cell_material(const vfo_problem *P, int ei, int ej, int ek) {
  cellmat m;
  int l = P->layer ? P->layer[ek] : 0;
  double E = P->E[l], nu = P->nu[l];
  if (P->cellE) E = P->cellE[((int64_t)ek * (P->ny - 1) + ej) * (P->nx - 1) + ei];
  m.lambda = E * nu / (1. + nu) / (1. - 2. * nu);
  m.mu = E / (1. + nu) * .5;
  m.alpha = P->alpha[l];
  m.beta = P->beta[l];
  m.Gc = P->Gc[l];
  return m;
}

static double atCv(const vfo_problem *P) { return P->atnum == 1 ? 2. / 3. : .5; } /* VFCommon.c:482-492 */

/* ------------------------------------------------------------------------ */
/* VFCartFEElement1DInit (VFCartFE.c:90-116) and VFCartFEElement3DInit
 * (VFCartFE.c:216-269): 3-point Gauss per axis, tensor product, g = gi+3gj+9gk. */
typedef struct {
  double w[27];
  double phi[8][27];
  double dphi[8][3][27];
} etab;

static void tables1d(double l, double w[3], double phi[2][3], double dphi[2][3]) {
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
}

static void etab_init(etab *e, double hx, double hy, double hz) {
  double wx[3], wy[3], wz[3], px[2][3], py[2][3], pz[2][3], dx[2][3], dy[2][3], dz[2][3];
  tables1d(hx, wx, px, dx);
  tables1d(hy, wy, py, dy);
  tables1d(hz, wz, pz, dz);
  for (int gk = 0, g = 0; gk < 3; gk++)
    for (int gj = 0; gj < 3; gj++)
      for (int gi = 0; gi < 3; gi++, g++) e->w[g] = wz[gk] * wy[gj] * wx[gi];
  for (int gk = 0, g = 0; gk < 3; gk++)
    for (int gj = 0; gj < 3; gj++)
      for (int gi = 0; gi < 3; gi++, g++)
        for (int k = 0; k < 2; k++)
          for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
              int a = i + 2 * j + 4 * k;
              e->phi[a][g] = pz[k][gk] * py[j][gj] * px[i][gi];
              e->dphi[a][0][g] = pz[k][gk] * py[j][gj] * dx[i][gi];
              e->dphi[a][1][g] = pz[k][gk] * dy[j][gj] * px[i][gi];
              e->dphi[a][2][g] = dz[k][gk] * py[j][gj] * px[i][gi];
            }
}

int vfo_tables(double hx, double hy, double hz, double w[27], double phi[8 * 27],
               double dphi[8 * 3 * 27]) {
  etab e;
  etab_init(&e, hx, hy, hz);
  memcpy(w, e.w, sizeof e.w);
  memcpy(phi, e.phi, sizeof e.phi);
  memcpy(dphi, e.dphi, sizeof e.dphi);
  return 0;
}

static void cell_nodes(const vfo_problem *P, int ei, int ej, int ek, int64_t n[8]) {
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) n[i + 2 * j + 4 * k] = NODE(P, ei + i, ej + j, ek + k);
}

/* ------------------------------------------------------------------------ */
/* Dirichlet BC, VecApplyDirichletBC / ResidualApplyDirichletBC precedence
 * (VFCartFE.c:493-998): faces X0,X1,Y0,Y1,Z0,Z1 in order (later wins), then the
 * 8 vertices in the order the reference applies them. */
int vfo_bc_build(int nx, int ny, int nz, int dof, const int *face, const int *vertex,
                 const double *bcu, uint8_t *mask, double *value) {
  int64_t N = (int64_t)nx * ny * nz;
  memset(mask, 0, (size_t)(N * dof));
  for (int64_t q = 0; q < N * dof; q++) value[q] = 0.;
#define SETBC(ii, jj, kk, type)                                                  \
  do {                                                                           \
    int64_t q_ = (((int64_t)(kk) * ny + (jj)) * nx + (ii)) * dof + c;            \
    mask[q_] = 1;                                                                \
    value[q_] = (type) == VFO_ZERO ? 0. : (type) == VFO_ONE ? 1. : (bcu ? bcu[q_] : 0.); \
  } while (0)
  for (int c = 0; c < dof; c++) {
    const int *f = face + 6 * c;
    for (int fc = 0; fc < 6; fc++) {
      int t = f[fc];
      if (t == VFO_NONE) continue;
      if (fc < 2) {
        int i = fc == 0 ? 0 : nx - 1;
        for (int k = 0; k < nz; k++)
          for (int j = 0; j < ny; j++) SETBC(i, j, k, t);
      } else if (fc < 4) {
        int j = fc == 2 ? 0 : ny - 1;
        for (int k = 0; k < nz; k++)
          for (int i = 0; i < nx; i++) SETBC(i, j, k, t);
      } else {
        int k = fc == 4 ? 0 : nz - 1;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) SETBC(i, j, k, t);
      }
    }
    /* VERTEX enum: X0Y0Z0,X1Y0Z0,X0Y1Z0,X1Y1Z0,X0Y0Z1,X1Y0Z1,X0Y1Z1,X1Y1Z1 (VFCartFE.h:121-130);
     * applied in the order X0Y0Z0, X0Y0Z1, X0Y1Z0, X0Y1Z1, X1Y0Z0, X1Y0Z1, X1Y1Z0, X1Y1Z1
     * (VFCartFE.c:950-972). */
    static const int order[8] = {0, 4, 2, 6, 1, 5, 3, 7};
    for (int o = 0; o < 8; o++) {
      int vtx = order[o];
      int t = vertex[8 * c + vtx];
      if (t == VFO_NONE) continue;
      int i = (vtx & 1) ? nx - 1 : 0, j = (vtx & 2) ? ny - 1 : 0, k = (vtx & 4) ? nz - 1 : 0;
      SETBC(i, j, k, t);
    }
  }
#undef SETBC
  return 0;
}

/* ------------------------------------------------------------------------ */
/* VF_BilinearFormU3D_local (VFMech.c:227-290). */
static void u_element_matrix(const etab *e, const cellmat *m, double eta, const double v8[8],
                             double K[576]) {
  double s[27];
  for (int g = 0; g < 27; g++) s[g] = 0.;
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) s[g] += v8[a] * e->phi[a][g];
  for (int g = 0; g < 27; g++) s[g] = s[g] * s[g] + eta;
  for (int l = 0; l < 576; l++) K[l] = 0;
  int l = 0;
  for (int a = 0; a < 8; a++)
    for (int c1 = 0; c1 < 3; c1++)
      for (int b = 0; b < 8; b++)
        for (int c2 = 0; c2 < 3; c2++, l++)
          for (int g = 0; g < 27; g++) {
            double mg = m->lambda * s[g] * e->dphi[a][c1][g] * e->dphi[b][c2][g];
            mg += m->mu * s[g] * e->dphi[a][c2][g] * e->dphi[b][c1][g];
            if (c1 == c2)
              mg += m->mu * s[g] *
                    (e->dphi[a][0][g] * e->dphi[b][0][g] + e->dphi[a][1][g] * e->dphi[b][1][g] +
                     e->dphi[a][2][g] * e->dphi[b][2][g]);
            K[l] += e->w[g] * mg;
          }
}

int vfo_u_element_matrix(const vfo_problem *P, int ei, int ej, int ek, const double *v,
                         double K[576]) {
  double hx, hy, hz, v8[8];
  int64_t n[8];
  etab e;
  cell_h(P, ei, ej, ek, &hx, &hy, &hz);
  etab_init(&e, hx, hy, hz);
  cell_nodes(P, ei, ej, ek, n);
  for (int a = 0; a < 8; a++) v8[a] = v[n[a]];
  cellmat m = cell_material(P, ei, ej, ek);
  u_element_matrix(&e, &m, P->eta, v8, K);
  return 0;
}

/* VF_GradientUThermoPoro3D_local (VFMech.c:386-447). */
static void u_rhs_thermoporo(const etab *e, const cellmat *m, double eta, const double th8[8],
                             const double p8[8], const double v8[8], double rl[24]) {
  double coefalpha = (3. * m->lambda + 2. * m->mu) * m->alpha, beta = m->beta;
  double te[27], pe[27], ve[27];
  for (int g = 0; g < 27; g++) te[g] = pe[g] = ve[g] = 0.;
  for (int g = 0; g < 27; g++)
    for (int a = 0; a < 8; a++) {
      te[g] += e->phi[a][g] * th8[a];
      pe[g] += e->phi[a][g] * p8[a];
      ve[g] += e->phi[a][g] * v8[a];
    }
  for (int g = 0; g < 27; g++)
    for (int a = 0, l = 0; a < 8; a++)
      for (int c = 0; c < 3; c++, l++)
        rl[l] += e->w[g] * e->dphi[a][c][g] *
                 (coefalpha * te[g] * (ve[g] * ve[g] + eta) + beta * pe[g] * ve[g]);
}

/* VF_GradientUCrackPressure3D_local (VFMech.c:533-589). */
static void u_rhs_crackpressure(const etab *e, const double p8[8], const double v8[8],
                                double rl[24]) {
  double pe[27], gv[3][27];
  for (int g = 0; g < 27; g++) {
    pe[g] = 0;
    for (int c = 0; c < 3; c++) gv[c][g] = 0.;
  }
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) {
      pe[g] += e->phi[a][g] * p8[a];
      for (int c = 0; c < 3; c++) gv[c][g] += e->dphi[a][c][g] * v8[a];
    }
  for (int a = 0, l = 0; a < 8; a++)
    for (int c = 0; c < 3; c++, l++)
      for (int g = 0; g < 27; g++) rl[l] += e->w[g] * pe[g] * gv[c][g] * e->phi[a][g];
}

/* VF_BilinearFormUNoCompression3D_local (VFMech.c:299-376): at the Gauss points
 * where tr(eps(u0)) < 0 (UNILATERAL_THRES = 0, VFMech.c:6) the spherical part keeps
 * kappa (1 + eta) instead of kappa s; the deviatoric part is always degraded. */
static void u_element_matrix_nc(const etab *e, const cellmat *m, double eta, const double v8[8],
                                const double u8[8][3], double K[576]) {
  const double kappa = m->lambda + 2. * m->mu / 3.;
  double s[27], tr[27];
  for (int g = 0; g < 27; g++) s[g] = tr[g] = 0.;
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) {
      s[g] += v8[a] * e->phi[a][g];
      tr[g] += e->dphi[a][0][g] * u8[a][0] + e->dphi[a][1][g] * u8[a][1] +
               e->dphi[a][2][g] * u8[a][2];
    }
  for (int g = 0; g < 27; g++) s[g] = s[g] * s[g] + eta;
  for (int l = 0; l < 576; l++) K[l] = 0;
  int l = 0;
  for (int a = 0; a < 8; a++)
    for (int c1 = 0; c1 < 3; c1++)
      for (int b = 0; b < 8; b++)
        for (int c2 = 0; c2 < 3; c2++, l++)
          for (int g = 0; g < 27; g++) {
            double mg = (tr[g] < 0. ? kappa * (1. + eta) : kappa * s[g]) * e->dphi[a][c1][g] *
                        e->dphi[b][c2][g];
            mg -= 2. * m->mu * s[g] * e->dphi[a][c1][g] * e->dphi[b][c2][g] / 3.;
            mg += m->mu * s[g] * e->dphi[a][c2][g] * e->dphi[b][c1][g];
            if (c1 == c2)
              mg += m->mu * s[g] *
                    (e->dphi[a][0][g] * e->dphi[b][0][g] + e->dphi[a][1][g] * e->dphi[b][1][g] +
                     e->dphi[a][2][g] * e->dphi[b][2][g]);
            K[l] += e->w[g] * mg;
          }
}

/* VF_GradientUThermoPoroNoCompression3D_local (VFMech.c:456-524): where
 * tr(eps(u0)) < 0 the thermal term is not degraded and the pore pressure is not
 * multiplied by v. */
static void u_rhs_thermoporo_nc(const etab *e, const cellmat *m, double eta, const double th8[8],
                                const double p8[8], const double v8[8], const double u8[8][3],
                                double rl[24]) {
  double coefalpha = (3. * m->lambda + 2. * m->mu) * m->alpha, beta = m->beta;
  double te[27], pe[27], ve[27], tr[27];
  for (int g = 0; g < 27; g++) te[g] = pe[g] = ve[g] = tr[g] = 0.;
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) {
      te[g] += e->phi[a][g] * th8[a];
      pe[g] += e->phi[a][g] * p8[a];
      ve[g] += e->phi[a][g] * v8[a];
      tr[g] += e->dphi[a][0][g] * u8[a][0] + e->dphi[a][1][g] * u8[a][1] +
               e->dphi[a][2][g] * u8[a][2];
    }
  for (int g = 0; g < 27; g++)
    for (int a = 0, l = 0; a < 8; a++)
      for (int c = 0; c < 3; c++, l++) {
        if (tr[g] < 0.)
          rl[l] += e->w[g] * e->dphi[a][c][g] * (coefalpha * te[g] * (1. + eta) + beta * pe[g]);
        else
          rl[l] += e->w[g] * e->dphi[a][c][g] *
                   (coefalpha * te[g] * (ve[g] * ve[g] + eta) + beta * pe[g] * ve[g]);
      }
}

/* u at the 8 nodes of a cell, zeros for u = NULL */
static void gather_u8z(const vfo_problem *P, int ei, int ej, int ek, const double *u,
                       double u8[8][3]) {
  int64_t n[8];
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) n[i + 2 * j + 4 * k] = NODE(P, ei + i, ej + j, ek + k);
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++) u8[a][c] = u ? u[3 * n[a] + c] : 0.;
}

/* The U element matrix of the problem's unilateral model at u0. */
static void u_element_matrix_any(const vfo_problem *P, int ei, int ej, int ek, const etab *e,
                                 const cellmat *m, const double v8[8], const double *u0,
                                 double K[576]) {
  if (P->unilateral) {
    double u8[8][3];
    gather_u8z(P, ei, ej, ek, u0, u8);
    u_element_matrix_nc(e, m, P->eta, v8, u8, K);
  } else {
    u_element_matrix(e, m, P->eta, v8, K);
  }
}

static void u_rhs_thermoporo_any(const vfo_problem *P, int ei, int ej, int ek, const etab *e,
                                 const cellmat *m, const double th8[8], const double p8[8],
                                 const double v8[8], const double *u0, double rl[24]) {
  if (P->unilateral) {
    double u8[8][3];
    gather_u8z(P, ei, ej, ek, u0, u8);
    u_rhs_thermoporo_nc(e, m, P->eta, th8, p8, v8, u8, rl);
  } else {
    u_rhs_thermoporo(e, m, P->eta, th8, p8, v8, rl);
  }
}

static void gather_cell(const vfo_problem *P, int ei, int ej, int ek, const double *v,
                        const double *theta, const double *thetaRef, const double *p,
                        double v8[8], double th8[8], double p8[8]) {
  int64_t n[8];
  cell_nodes(P, ei, ej, ek, n);
  for (int a = 0; a < 8; a++) {
    if (v8) v8[a] = v[n[a]];
    if (th8) th8[a] = theta ? theta[n[a]] - (thetaRef ? thetaRef[n[a]] : 0.) : 0.;
    if (p8) p8[a] = p ? p[n[a]] : 0.;
  }
}

/* VF_UResidual (VFMech.c:1456-1887) without in-situ tractions: element loop in
 * the reference's order, F += K_e u_e then F -= (thermo-poro + crack pressure),
 * then ResidualApplyDirichletBC (F = u - ubc on BC rows). */
/* ------------------------------------------------------------------------ */
/* In-situ tractions.  Face order and the stress component / sign of each face
 * component (VFMech.c:1630-1848): t_c = dir * s_comp(z) with s linear in z
 * between insitumin (z = BBmin = 0) and insitumax (z = BBmax = lz). */
static const int insitu_comp[6][3] = {{0, 5, 4}, {0, 5, 4}, {5, 1, 3},
                                      {5, 1, 3}, {4, 3, 2}, {4, 3, 2}};
static const double insitu_dir[6] = {-1., 1., -1., 1., -1., 1.};
enum { F_X0 = 0, F_X1, F_Y0, F_Y1, F_Z0, F_Z1 };

static double insitu_traction(const vfo_problem *P, int face, int c, double z) {
  const int s = insitu_comp[face][c];
  return insitu_dir[face] *
         (P->insitumin[s] + (z - 0.) / (P->lz - 0.) * (P->insitumax[s] - P->insitumin[s]));
}

/* Local node (i,j,k) of a cell projected onto the face's node layer: the face
 * layer index replaces the normal-direction index (VFMech.c:610-700). */
static void face_project(int face, int i, int j, int k, int *pi, int *pj, int *pk) {
  *pi = i;
  *pj = j;
  *pk = k;
  if (face == F_X0) *pi = 0;
  if (face == F_X1) *pi = 1;
  if (face == F_Y0) *pj = 0;
  if (face == F_Y1) *pj = 1;
  if (face == F_Z0) *pk = 0;
  if (face == F_Z1) *pk = 1;
}

/* VF_GradientUInSituStresses3D_local for one boundary cell and face, added to the
 * face nodes as the reference does (every local row lands on the face layer).
 * Components with a Dirichlet BC on the face get no traction (their rows are
 * replaced by the BC; the reference leaves stale values there). */
static void insitu_load_cell(const vfo_problem *P, int ei, int ej, int ek, int face, double sgn,
                             double *f) {
  double hx, hy, hz;
  etab e;
  cell_h(P, ei, ej, ek, &hx, &hy, &hz);
  etab_init(&e, hx, hy, hz);
  const double hn = face <= F_X1 ? hx : (face <= F_Y1 ? hy : hz);
  double t[8][3], felem[3][27], rl[8][3];
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) {
        int pi, pj, pk;
        face_project(face, i, j, k, &pi, &pj, &pk);
        const double z = coord(ek + pk, P->lz, P->nz);
        for (int c = 0; c < 3; c++)
          t[i + 2 * j + 4 * k][c] = P->insitu_free[face][c] ? insitu_traction(P, face, c, z) : 0.;
      }
  for (int c = 0; c < 3; c++)
    for (int g = 0; g < 27; g++) felem[c][g] = 0.;
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++)
      for (int g = 0; g < 27; g++) felem[c][g] += e.phi[a][g] * t[a][c] / hn;
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++) {
      rl[a][c] = 0.;
      for (int g = 0; g < 27; g++) rl[a][c] += e.w[g] * e.phi[a][g] * felem[c][g];
    }
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) {
        int pi, pj, pk;
        face_project(face, i, j, k, &pi, &pj, &pk);
        const int64_t q = NODE(P, ei + pi, ej + pj, ek + pk);
        for (int c = 0; c < 3; c++) f[3 * q + c] += sgn * rl[i + 2 * j + 4 * k][c];
      }
}

/* The in-situ part of one cell's residual contribution, faces in the reference's
 * order (VFMech.c:1630-1848); sgn = +1 adds the load to f, -1 subtracts it from F. */
static void insitu_cell(const vfo_problem *P, int ei, int ej, int ek, double sgn, double *f) {
  const int ncx = P->nx - 1, ncy = P->ny - 1, ncz = P->nz - 1;
  if (ek == 0) insitu_load_cell(P, ei, ej, ek, F_Z0, sgn, f);
  if (ek == ncz - 1) insitu_load_cell(P, ei, ej, ek, F_Z1, sgn, f);
  if (ej == 0) insitu_load_cell(P, ei, ej, ek, F_Y0, sgn, f);
  if (ej == ncy - 1) insitu_load_cell(P, ei, ej, ek, F_Y1, sgn, f);
  if (ei == 0) insitu_load_cell(P, ei, ej, ek, F_X0, sgn, f);
  if (ei == ncx - 1) insitu_load_cell(P, ei, ej, ek, F_X1, sgn, f);
}

static void insitu_load(const vfo_problem *P, double *f) {
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) insitu_cell(P, ei, ej, ek, 1., f);
}

/* VF_InSituStressWork3D_local over the faces as VF_UEnergy3D visits them
 * (VFMech.c:1238-1400): X0/Y0/Z0 at the first cell layer; X1/Y1/Z1 at cell layer
 * ncells-2 (the reference compares the cell index with the cell count minus 2), so
 * u and the traction are taken at the node layer one inside the box. */
static double insitu_work_cell(const vfo_problem *P, const double *u, int ei, int ej, int ek,
                               int face) {
  double hx, hy, hz;
  etab e;
  cell_h(P, ei, ej, ek, &hx, &hy, &hz);
  etab_init(&e, hx, hy, hz);
  const double hn = face <= F_X1 ? hx : (face <= F_Y1 ? hy : hz);
  double ue[3][27], fe[3][27];
  for (int c = 0; c < 3; c++)
    for (int g = 0; g < 27; g++) ue[c][g] = fe[c][g] = 0.;
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) {
        int pi, pj, pk;
        face_project(face, i, j, k, &pi, &pj, &pk);
        const int64_t q = NODE(P, ei + pi, ej + pj, ek + pk);
        const double z = coord(ek + pk, P->lz, P->nz);
        const int a = i + 2 * j + 4 * k;
        for (int c = 0; c < 3; c++) {
          const double t = P->insitu_free[face][c] ? insitu_traction(P, face, c, z) : 0.;
          for (int g = 0; g < 27; g++) {
            ue[c][g] += e.phi[a][g] * u[3 * q + c] / hn;
            fe[c][g] += e.phi[a][g] * t;
          }
        }
      }
  double w = 0.;
  for (int c = 0; c < 3; c++)
    for (int g = 0; g < 27; g++) w += e.w[g] * ue[c][g] * fe[c][g];
  return w;
}

int vfo_insitu_work(const vfo_problem *P, const double *u, double *work) {
  const int ncx = P->nx - 1, ncy = P->ny - 1, ncz = P->nz - 1;
  double w = 0.;
  if (P->hasInsitu)
    for (int ek = 0; ek < ncz; ek++)
      for (int ej = 0; ej < ncy; ej++)
        for (int ei = 0; ei < ncx; ei++) {
          if (ek == 0) w += insitu_work_cell(P, u, ei, ej, ek, F_Z0);
          if (ek == ncz - 2) w += insitu_work_cell(P, u, ei, ej, ek, F_Z1);
          if (ej == 0) w += insitu_work_cell(P, u, ei, ej, ek, F_Y0);
          if (ej == ncy - 2) w += insitu_work_cell(P, u, ei, ej, ek, F_Y1);
          if (ei == 0) w += insitu_work_cell(P, u, ei, ej, ek, F_X0);
          if (ei == ncx - 2) w += insitu_work_cell(P, u, ei, ej, ek, F_X1);
        }
  *work = w;
  return 0;
}

int vfo_u_residual_ref(const vfo_problem *P, const double *u, const double *v,
                       const double *theta, const double *thetaRef, const double *p,
                       const uint8_t *bcmask, const double *bcval, double *F) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < 3 * N; q++) F[q] = 0.;
  double K[576], rl[24], v8[8], th8[8], p8[8], hx, hy, hz;
  int64_t n[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        cell_nodes(P, ei, ej, ek, n);
        gather_cell(P, ei, ej, ek, v, theta, thetaRef, p, v8, th8, p8);
        u_element_matrix_any(P, ei, ej, ek, &e, &m, v8, u, K);
        int l = 0;
        for (int a = 0; a < 8; a++)
          for (int c1 = 0; c1 < 3; c1++)
            for (int b = 0; b < 8; b++)
              for (int c2 = 0; c2 < 3; c2++, l++) F[3 * n[a] + c1] += K[l] * u[3 * n[b] + c2];
        for (l = 0; l < 24; l++) rl[l] = 0.;
        u_rhs_thermoporo_any(P, ei, ej, ek, &e, &m, th8, p8, v8, u, rl);
        if (P->hasCrackPressure) u_rhs_crackpressure(&e, p8, v8, rl);
        for (int a = 0, l2 = 0; a < 8; a++)
          for (int c = 0; c < 3; c++, l2++) F[3 * n[a] + c] -= rl[l2];
        if (P->hasInsitu) insitu_cell(P, ei, ej, ek, -1., F);
      }
  if (bcmask)
    for (int64_t q = 0; q < 3 * N; q++)
      if (bcmask[q]) F[q] = u[q] - bcval[q];
  return 0;
}

/* J x with the assembled element matrices (VF_UIJacobian, VFMech.c:1897-2029):
 * BC rows are identity, BC columns are kept (MatZeroRowsStencil, VFCartFE.c:1293). */
int vfo_u_apply_ref(const vfo_problem *P, const double *v, const double *x,
                    const uint8_t *bcmask, double *y) {
  return vfo_u_apply_ref_u(P, NULL, v, x, bcmask, y);
}

int vfo_u_apply_ref_u(const vfo_problem *P, const double *u0, const double *v, const double *x,
                      const uint8_t *bcmask, double *y) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < 3 * N; q++) y[q] = 0.;
  double K[576], hx, hy, hz, v8[8];
  int64_t n[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        cell_nodes(P, ei, ej, ek, n);
        for (int a = 0; a < 8; a++) v8[a] = v[n[a]];
        u_element_matrix_any(P, ei, ej, ek, &e, &m, v8, u0, K);
        int l = 0;
        for (int a = 0; a < 8; a++)
          for (int c1 = 0; c1 < 3; c1++)
            for (int b = 0; b < 8; b++)
              for (int c2 = 0; c2 < 3; c2++, l++) y[3 * n[a] + c1] += K[l] * x[3 * n[b] + c2];
      }
  if (bcmask)
    for (int64_t q = 0; q < 3 * N; q++)
      if (bcmask[q]) y[q] = x[q];
  return 0;
}

/* Matrix-free J x, per-Gauss-point form of the same bilinear form:
 * y_(a,c) = sum_g sum_d dphi_a,d(g) sigma_cd(g),
 * sigma = w s (lambda tr(G) I + mu (G + G^T)),  G_cd = sum_b dphi_b,d u_(b,c).
 * Elements are visited in 8 parity colours so the OpenMP scatter is race-free
 * and the result is independent of the thread count. */
int vfo_u_apply_mf(const vfo_problem *P, const double *v, const double *x,
                   const uint8_t *bcmask, double *y) {
  return vfo_u_apply_mf_u(P, NULL, v, x, bcmask, y);
}

/* NOCOMPRESSION: sigma = w [lambda' tr(G) I + s mu (G + G^T)] with
 * lambda' = kappa (1 + eta) - 2 mu s / 3 where tr(eps(u0)) < 0, else lambda s. */
int vfo_u_apply_mf_u(const vfo_problem *P, const double *u0, const double *v, const double *x,
                     const uint8_t *bcmask, double *y) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < 3 * N; q++) y[q] = 0.;
  int nex = P->nx - 1, ney = P->ny - 1, nez = P->nz - 1;
  if (P->nthreads > 0) {
#ifdef _OPENMP
    omp_set_num_threads(P->nthreads);
#endif
  }
  for (int color = 0; color < 8; color++) {
    int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    int hx_n = (nex - cx + 1) / 2, hy_n = (ney - cy + 1) / 2, hz_n = (nez - cz + 1) / 2;
    int64_t total = (int64_t)hx_n * hy_n * hz_n;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < total; t++) {
      int ei = cx + 2 * (int)(t % hx_n);
      int ej = cy + 2 * (int)((t / hx_n) % hy_n);
      int ek = cz + 2 * (int)(t / ((int64_t)hx_n * hy_n));
      double hx, hy, hz;
      etab e;
      cell_h(P, ei, ej, ek, &hx, &hy, &hz);
      etab_init(&e, hx, hy, hz);
      cellmat m = cell_material(P, ei, ej, ek);
      int64_t n[8];
      cell_nodes(P, ei, ej, ek, n);
      double ue[8][3], v8[8], ye[8][3], u08[8][3];
      for (int a = 0; a < 8; a++) {
        v8[a] = v[n[a]];
        for (int c = 0; c < 3; c++) {
          ue[a][c] = x[3 * n[a] + c];
          u08[a][c] = u0 ? u0[3 * n[a] + c] : 0.;
          ye[a][c] = 0.;
        }
      }
      const double kappa = m.lambda + 2. * m.mu / 3.;
      for (int g = 0; g < 27; g++) {
        double s = 0., tr0 = 0., G[3][3] = {{0}};
        for (int a = 0; a < 8; a++) {
          s += v8[a] * e.phi[a][g];
          for (int c = 0; c < 3; c++) {
            tr0 += e.dphi[a][c][g] * u08[a][c];
            for (int d = 0; d < 3; d++) G[c][d] += e.dphi[a][d][g] * ue[a][c];
          }
        }
        const double sv = s * s + P->eta;
        double ws = e.w[g] * sv;
        double tr = G[0][0] + G[1][1] + G[2][2], sg[3][3];
        const double lam_tr = (P->unilateral && tr0 < 0.)
                                  ? e.w[g] * (kappa * (1. + P->eta) - 2. * m.mu * sv / 3.) * tr
                                  : ws * m.lambda * tr;
        for (int c = 0; c < 3; c++)
          for (int d = 0; d < 3; d++)
            sg[c][d] = (c == d ? lam_tr : 0.) + ws * m.mu * (G[c][d] + G[d][c]);
        for (int a = 0; a < 8; a++)
          for (int c = 0; c < 3; c++)
            ye[a][c] += e.dphi[a][0][g] * sg[c][0] + e.dphi[a][1][g] * sg[c][1] +
                        e.dphi[a][2][g] * sg[c][2];
      }
      for (int a = 0; a < 8; a++)
        for (int c = 0; c < 3; c++) y[3 * n[a] + c] += ye[a][c];
    }
  }
  if (bcmask)
    for (int64_t q = 0; q < 3 * N; q++)
      if (bcmask[q]) y[q] = x[q];
  return 0;
}

/* f with F = K u - f: the thermo-poro and crack-pressure load vectors of
 * VF_UResidual (VFMech.c:1600-1626), summed in element order. */
int vfo_u_rhs(const vfo_problem *P, const double *v, const double *theta,
              const double *thetaRef, const double *p, double *f) {
  return vfo_u_rhs_u(P, NULL, v, theta, thetaRef, p, f);
}

int vfo_u_rhs_u(const vfo_problem *P, const double *u0, const double *v, const double *theta,
                const double *thetaRef, const double *p, double *f) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < 3 * N; q++) f[q] = 0.;
  double rl[24], v8[8], th8[8], p8[8], hx, hy, hz;
  int64_t n[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        cell_nodes(P, ei, ej, ek, n);
        gather_cell(P, ei, ej, ek, v, theta, thetaRef, p, v8, th8, p8);
        for (int l = 0; l < 24; l++) rl[l] = 0.;
        u_rhs_thermoporo_any(P, ei, ej, ek, &e, &m, th8, p8, v8, u0, rl);
        if (P->hasCrackPressure) u_rhs_crackpressure(&e, p8, v8, rl);
        for (int a = 0, l = 0; a < 8; a++)
          for (int c = 0; c < 3; c++, l++) f[3 * n[a] + c] += rl[l];
      }
  if (P->hasInsitu) insitu_load(P, f);
  return 0;
}

/* Diagonal of K(v) (the Jacobi preconditioner of KSPCG with -U_pc_type jacobi),
 * BC rows 1 as after MatZeroRowsStencil. */
int vfo_u_diag(const vfo_problem *P, const double *v, const uint8_t *bcmask, double *d) {
  return vfo_u_diag_u(P, NULL, v, bcmask, d);
}

int vfo_u_diag_u(const vfo_problem *P, const double *u0, const double *v, const uint8_t *bcmask,
                 double *d) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < 3 * N; q++) d[q] = 0.;
  double K[576], hx, hy, hz, v8[8];
  int64_t n[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        cell_nodes(P, ei, ej, ek, n);
        for (int a = 0; a < 8; a++) v8[a] = v[n[a]];
        u_element_matrix_any(P, ei, ej, ek, &e, &m, v8, u0, K);
        for (int a = 0; a < 8; a++)
          for (int c = 0; c < 3; c++) d[3 * n[a] + c] += K[(3 * a + c) * 24 + 3 * a + c];
      }
  if (bcmask)
    for (int64_t q = 0; q < 3 * N; q++)
      if (bcmask[q]) d[q] = 1.;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* CSR assembly of the DMDA AIJ matrix (box stencil, 3 dof: up to 81 nnz/row,
 * columns ascending) -- what PETSc's MatMult runs inside KSPCG. */
int64_t vfo_u_csr_nnz(const vfo_problem *P) {
  int64_t nnz = 0;
  for (int k = 0; k < P->nz; k++)
    for (int j = 0; j < P->ny; j++)
      for (int i = 0; i < P->nx; i++) {
        int cx = (i > 0) + 1 + (i < P->nx - 1), cy = (j > 0) + 1 + (j < P->ny - 1),
            cz = (k > 0) + 1 + (k < P->nz - 1);
        nnz += 3 * 3 * (int64_t)cx * cy * cz;
      }
  return nnz;
}

static int64_t csr_pos(const vfo_problem *P, const int64_t *rowptr, int i, int j, int k, int c1,
                       int di, int dj, int dk, int c2) {
  /* columns of row (i,j,k,c1): neighbours in (k,j,i) order then component */
  int x0 = i > 0 ? i - 1 : 0, x1 = i < P->nx - 1 ? i + 1 : i;
  int y0 = j > 0 ? j - 1 : 0, y1 = j < P->ny - 1 ? j + 1 : j;
  int z0 = k > 0 ? k - 1 : 0;
  int cx = x1 - x0 + 1, cy = y1 - y0 + 1;
  int ox = i + di - x0, oy = j + dj - y0, oz = k + dk - z0;
  int64_t row = 3 * NODE(P, i, j, k) + c1;
  return rowptr[row] + ((int64_t)(oz * cy + oy) * cx + ox) * 3 + c2;
}

int vfo_u_assemble_csr(const vfo_problem *P, const double *v, const uint8_t *bcmask,
                       int64_t *rowptr, int32_t *colidx, double *vals) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz, r = 0;
  rowptr[0] = 0;
  for (int k = 0; k < P->nz; k++)
    for (int j = 0; j < P->ny; j++)
      for (int i = 0; i < P->nx; i++)
        for (int c1 = 0; c1 < 3; c1++, r++) {
          int64_t pos = rowptr[r];
          for (int kk = k - 1; kk <= k + 1; kk++)
            for (int jj = j - 1; jj <= j + 1; jj++)
              for (int ii = i - 1; ii <= i + 1; ii++) {
                if (ii < 0 || jj < 0 || kk < 0 || ii >= P->nx || jj >= P->ny || kk >= P->nz)
                  continue;
                for (int c2 = 0; c2 < 3; c2++) {
                  colidx[pos] = (int32_t)(3 * NODE(P, ii, jj, kk) + c2);
                  vals[pos] = 0.;
                  pos++;
                }
              }
          rowptr[r + 1] = pos;
        }
  int nex = P->nx - 1, ney = P->ny - 1, nez = P->nz - 1;
  for (int color = 0; color < 8; color++) {
    int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    int hx_n = (nex - cx + 1) / 2, hy_n = (ney - cy + 1) / 2, hz_n = (nez - cz + 1) / 2;
    int64_t total = (int64_t)hx_n * hy_n * hz_n;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < total; t++) {
      int ei = cx + 2 * (int)(t % hx_n);
      int ej = cy + 2 * (int)((t / hx_n) % hy_n);
      int ek = cz + 2 * (int)(t / ((int64_t)hx_n * hy_n));
      double K[576];
      vfo_u_element_matrix(P, ei, ej, ek, v, K);
      int l = 0;
      for (int a = 0; a < 8; a++)
        for (int c1 = 0; c1 < 3; c1++)
          for (int b = 0; b < 8; b++)
            for (int c2 = 0; c2 < 3; c2++, l++) {
              int ai = a & 1, aj = (a >> 1) & 1, ak = a >> 2;
              int bi = b & 1, bj = (b >> 1) & 1, bk = b >> 2;
              int64_t pos = csr_pos(P, rowptr, ei + ai, ej + aj, ek + ak, c1, bi - ai, bj - aj,
                                    bk - ak, c2);
              vals[pos] += K[l];
            }
    }
  }
  if (bcmask)
    for (int64_t q = 0; q < 3 * N; q++)
      if (bcmask[q])
        for (int64_t pos = rowptr[q]; pos < rowptr[q + 1]; pos++)
          vals[pos] = colidx[pos] == q ? 1. : 0.;
  return 0;
}

int vfo_csr_spmv(int64_t nrows, const int64_t *rowptr, const int32_t *colidx,
                 const double *vals, const double *x, double *y, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < nrows; r++) {
    double s = 0.;
    for (int64_t pos = rowptr[r]; pos < rowptr[r + 1]; pos++) s += vals[pos] * x[colidx[pos]];
    y[r] = s;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* ElasticEnergyDensity3D_local (VFMech.c:32-106). */
static void elastic_energy_density(const etab *e, const cellmat *m, const double u8[8][3],
                                   const double th8[8], double W[27]) {
  double e11[27], e22[27], e33[27], e12[27], e23[27], e13[27];
  double lambda = m->lambda, mu = m->mu, alpha = m->alpha;
  for (int g = 0; g < 27; g++) e11[g] = e22[g] = e33[g] = e12[g] = e23[g] = e13[g] = W[g] = 0.;
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) {
      e11[g] += e->dphi[a][0][g] * u8[a][0] - alpha * e->phi[a][g] * th8[a];
      e22[g] += e->dphi[a][1][g] * u8[a][1] - alpha * e->phi[a][g] * th8[a];
      e33[g] += e->dphi[a][2][g] * u8[a][2] - alpha * e->phi[a][g] * th8[a];
      e12[g] += (e->dphi[a][0][g] * u8[a][1] + e->dphi[a][1][g] * u8[a][0]) * .5;
      e23[g] += (e->dphi[a][1][g] * u8[a][2] + e->dphi[a][2][g] * u8[a][1]) * .5;
      e13[g] += (e->dphi[a][0][g] * u8[a][2] + e->dphi[a][2][g] * u8[a][0]) * .5;
    }
  for (int g = 0; g < 27; g++) {
    double s11 = (lambda + 2. * mu) * e11[g] + lambda * e22[g] + lambda * e33[g];
    double s22 = lambda * e11[g] + (lambda + 2. * mu) * e22[g] + lambda * e33[g];
    double s33 = lambda * e11[g] + lambda * e22[g] + (lambda + 2. * mu) * e33[g];
    double s12 = 2. * mu * e12[g], s23 = 2. * mu * e23[g], s13 = 2. * mu * e13[g];
    W[g] = (s11 * e11[g] + s22 * e22[g] + s33 * e33[g]) * .5 + s12 * e12[g] + s23 * e23[g] +
           s13 * e13[g];
  }
}

/* ElasticEnergyDensitySphericalDeviatoricNoCompression3D_local (VFMech.c:115-218):
 * W = sigma(eps - e0) : eps (the strain itself, not eps - e0, on the right), and the
 * coupling uses S + D = W - (kappa/2) tr^2 where tr < 0, W elsewhere
 * (kappa = lambda + 2 mu / 3). */
static void elastic_energy_density_nc(const etab *e, const cellmat *m, const double u8[8][3],
                                      const double th8[8], double W[27]) {
  double e11[27], e22[27], e33[27], e12[27], e23[27], e13[27], e0[27];
  double lambda = m->lambda, mu = m->mu, alpha = m->alpha, kappa = lambda + 2. * mu / 3.;
  for (int g = 0; g < 27; g++)
    e11[g] = e22[g] = e33[g] = e12[g] = e23[g] = e13[g] = e0[g] = W[g] = 0.;
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) {
      e11[g] += e->dphi[a][0][g] * u8[a][0];
      e22[g] += e->dphi[a][1][g] * u8[a][1];
      e33[g] += e->dphi[a][2][g] * u8[a][2];
      e12[g] += (e->dphi[a][0][g] * u8[a][1] + e->dphi[a][1][g] * u8[a][0]) * .5;
      e23[g] += (e->dphi[a][1][g] * u8[a][2] + e->dphi[a][2][g] * u8[a][1]) * .5;
      e13[g] += (e->dphi[a][0][g] * u8[a][2] + e->dphi[a][2][g] * u8[a][0]) * .5;
      e0[g] += alpha * e->phi[a][g] * th8[a];
    }
  for (int g = 0; g < 27; g++) {
    double s11 = (lambda + 2. * mu) * (e11[g] - e0[g]) + lambda * (e22[g] - e0[g]) +
                 lambda * (e33[g] - e0[g]);
    double s22 = lambda * (e11[g] - e0[g]) + (lambda + 2. * mu) * (e22[g] - e0[g]) +
                 lambda * (e33[g] - e0[g]);
    double s33 = lambda * (e11[g] - e0[g]) + lambda * (e22[g] - e0[g]) +
                 (lambda + 2. * mu) * (e33[g] - e0[g]);
    double s12 = 2. * mu * e12[g], s23 = 2. * mu * e23[g], s13 = 2. * mu * e13[g];
    double Wf = (s11 * e11[g] + s22 * e22[g] + s33 * e33[g]) * .5 + s12 * e12[g] +
                s23 * e23[g] + s13 * e13[g];
    double tr = e11[g] + e22[g] + e33[g];
    double S = tr < 0. ? 0. : kappa * tr * tr * .5;
    double D = Wf - kappa * tr * tr * .5;
    W[g] = S + D;
  }
}

/* VF_BilinearFormVAT1/AT23D_local + VF_BilinearFormVCoupling3D_local
 * (VFMech.c:2040-2115; NOCOMPRESSION: VF_BilinearFormVCouplingNoCompression3D_local,
 * VFMech.c:2125-2153), accumulated in the order VF_VResidual uses. */
static void v_element_matrix(const vfo_problem *P, const etab *e, const cellmat *m,
                             const double u8[8][3], const double th8[8], double K[64]) {
  double coef = m->Gc / atCv(P) * .5, eps = P->epsilon, W[27];
  for (int l = 0; l < 64; l++) K[l] = 0.;
  for (int a = 0, l = 0; a < 8; a++)
    for (int b = 0; b < 8; b++, l++)
      for (int g = 0; g < 27; g++) {
        double dd = e->dphi[a][0][g] * e->dphi[b][0][g] + e->dphi[a][1][g] * e->dphi[b][1][g] +
                    e->dphi[a][2][g] * e->dphi[b][2][g];
        if (P->atnum == 1)
          K[l] += coef * e->w[g] * dd * eps;
        else
          K[l] += coef * e->w[g] * (e->phi[a][g] * e->phi[b][g] / eps + dd * eps);
      }
  if (P->unilateral)
    elastic_energy_density_nc(e, m, u8, th8, W);
  else
    elastic_energy_density(e, m, u8, th8, W);
  for (int a = 0, l = 0; a < 8; a++)
    for (int b = 0; b < 8; b++, l++)
      for (int g = 0; g < 27; g++) K[l] += e->w[g] * e->phi[a][g] * e->phi[b][g] * W[g] * 2.;
}

static void gather_u8(const vfo_problem *P, int ei, int ej, int ek, const double *u,
                      double u8[8][3]) {
  int64_t n[8];
  cell_nodes(P, ei, ej, ek, n);
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++) u8[a][c] = u[3 * n[a] + c];
}

int vfo_v_element_matrix(const vfo_problem *P, int ei, int ej, int ek, const double *u,
                         const double *theta, const double *thetaRef, double K[64]) {
  double hx, hy, hz, u8[8][3], th8[8];
  etab e;
  cell_h(P, ei, ej, ek, &hx, &hy, &hz);
  etab_init(&e, hx, hy, hz);
  cellmat m = cell_material(P, ei, ej, ek);
  gather_u8(P, ei, ej, ek, u, u8);
  gather_cell(P, ei, ej, ek, NULL, theta, thetaRef, NULL, NULL, th8, NULL);
  v_element_matrix(P, &e, &m, u8, th8, K);
  return 0;
}

/* VF_ResidualVAT1/AT23D_local (VFMech.c:2350-2384). */
static void v_rhs_at(const vfo_problem *P, const etab *e, const cellmat *m, double rl[8]) {
  double coef = m->Gc / atCv(P) / P->epsilon * (P->atnum == 1 ? .25 : .5);
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) rl[a] += e->w[g] * e->phi[a][g] * coef;
}

/* VF_ResidualVCrackPressure3D_local (VFMech.c:2294-2341). */
static void v_rhs_crackpressure(const etab *e, const double u8[8][3], const double p8[8],
                                double rl[8]) {
  double pe[27], ue[3][27];
  for (int g = 0; g < 27; g++) {
    pe[g] = 0;
    for (int c = 0; c < 3; c++) ue[c][g] = 0.;
  }
  for (int a = 0; a < 8; a++)
    for (int g = 0; g < 27; g++) {
      pe[g] += e->phi[a][g] * p8[a];
      for (int c = 0; c < 3; c++) ue[c][g] += e->phi[a][g] * u8[a][c];
    }
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 3; c++)
      for (int g = 0; g < 27; g++) rl[a] += e->w[g] * pe[g] * ue[c][g] * e->dphi[a][c][g];
}

/* b with F_V = K_V v - b (AT linear term + crack pressure term). */
int vfo_v_rhs(const vfo_problem *P, const double *u, const double *p, double *b) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < N; q++) b[q] = 0.;
  double hx, hy, hz, u8[8][3], p8[8], rl[8];
  int64_t n[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        cell_nodes(P, ei, ej, ek, n);
        gather_u8(P, ei, ej, ek, u, u8);
        gather_cell(P, ei, ej, ek, NULL, NULL, NULL, p, NULL, NULL, p8);
        for (int a = 0; a < 8; a++) rl[a] = 0.;
        v_rhs_at(P, &e, &m, rl);
        if (P->hasCrackPressure) v_rhs_crackpressure(&e, u8, p8, rl);
        for (int a = 0; a < 8; a++) b[n[a]] += rl[a];
      }
  return 0;
}

/* VF_VResidual (VFMech.c:2687-2879), including quirk Q1: the thermo-poro
 * residual of VF_ResidualVThermoPoro3D_local is overwritten (VFMech.c:2809-2810)
 * and never reaches F; AT2 irreversibility zeroes F where VIrrev <= irrevtol
 * (VF_IrrevApplyEQVec, VFMech.c:2597-2628); V BC rows give F = v - bc. */
int vfo_v_residual_ref(const vfo_problem *P, const double *u, const double *v,
                       const double *theta, const double *thetaRef, const double *p,
                       const double *virrev, const uint8_t *bcmask, const double *bcval,
                       double *F) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < N; q++) F[q] = 0.;
  double hx, hy, hz, u8[8][3], th8[8], p8[8], rl[8], K[64];
  int64_t n[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        cell_nodes(P, ei, ej, ek, n);
        gather_u8(P, ei, ej, ek, u, u8);
        gather_cell(P, ei, ej, ek, NULL, theta, thetaRef, p, NULL, th8, p8);
        v_element_matrix(P, &e, &m, u8, th8, K);
        for (int a = 0; a < 8; a++) {
          rl[a] = 0.;
          for (int b = 0; b < 8; b++) rl[a] -= K[a * 8 + b] * v[n[b]];
        }
        v_rhs_at(P, &e, &m, rl);
        if (P->hasCrackPressure) v_rhs_crackpressure(&e, u8, p8, rl);
        for (int a = 0; a < 8; a++) F[n[a]] -= rl[a];
      }
  if (P->atnum == 2 && virrev)
    for (int64_t q = 0; q < N; q++)
      if (virrev[q] <= P->irrevtol) F[q] = 0.;
  if (bcmask)
    for (int64_t q = 0; q < N; q++)
      if (bcmask[q]) F[q] = v[q] - bcval[q];
  return 0;
}

static uint8_t v_fixed(const vfo_problem *P, const double *virrev, const uint8_t *bcmask,
                       int64_t q) {
  if (bcmask && bcmask[q]) return 1;
  if (P->atnum == 2 && virrev && virrev[q] <= P->irrevtol) return 1;
  return 0;
}

/* J_V x: MatApplyDirichletBCRowCol (VFCartFE.c:1305-1454) and, for AT2,
 * VF_IrrevApplyEQMat (VFMech.c:2637-2682) make those rows and columns identity. */
int vfo_v_apply(const vfo_problem *P, const double *u, const double *theta,
                const double *thetaRef, const double *virrev, const uint8_t *bcmask,
                const double *x, double *y) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < N; q++) y[q] = 0.;
  int nex = P->nx - 1, ney = P->ny - 1, nez = P->nz - 1;
  for (int color = 0; color < 8; color++) {
    int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    int hx_n = (nex - cx + 1) / 2, hy_n = (ney - cy + 1) / 2, hz_n = (nez - cz + 1) / 2;
    int64_t total = (int64_t)hx_n * hy_n * hz_n;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < total; t++) {
      int ei = cx + 2 * (int)(t % hx_n);
      int ej = cy + 2 * (int)((t / hx_n) % hy_n);
      int ek = cz + 2 * (int)(t / ((int64_t)hx_n * hy_n));
      double K[64];
      int64_t n[8];
      vfo_v_element_matrix(P, ei, ej, ek, u, theta, thetaRef, K);
      cell_nodes(P, ei, ej, ek, n);
      double xe[8];
      for (int b = 0; b < 8; b++) xe[b] = v_fixed(P, virrev, bcmask, n[b]) ? 0. : x[n[b]];
      for (int a = 0; a < 8; a++) {
        double s = 0.;
        for (int b = 0; b < 8; b++) s += K[a * 8 + b] * xe[b];
        y[n[a]] += s;
      }
    }
  }
  for (int64_t q = 0; q < N; q++)
    if (v_fixed(P, virrev, bcmask, q)) y[q] = x[q];
  return 0;
}

int vfo_v_diag(const vfo_problem *P, const double *u, const double *theta,
               const double *thetaRef, const double *virrev, const uint8_t *bcmask,
               double *d) {
  int64_t N = (int64_t)P->nx * P->ny * P->nz;
  for (int64_t q = 0; q < N; q++) d[q] = 0.;
  double K[64];
  int64_t n[8];
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        vfo_v_element_matrix(P, ei, ej, ek, u, theta, thetaRef, K);
        cell_nodes(P, ei, ej, ek, n);
        for (int a = 0; a < 8; a++) d[n[a]] += K[a * 9];
      }
  for (int64_t q = 0; q < N; q++)
    if (v_fixed(P, virrev, bcmask, q)) d[q] = 1.;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* VF_UEnergy3D (VFMech.c:1111-1427) without in-situ work: per element
 * VF_ElasticEnergy3D_local (VFMech.c:725-809, quirk Q2: v^2(1+eta) on the
 * deviatoric part) and VF_PressureWork3D_local (VFMech.c:920-974). */
int vfo_u_energy(const vfo_problem *P, const double *u, const double *v,
                 const double *theta, const double *thetaRef, const double *p,
                 double out[2]) {
  double myE = 0., myPW = 0., hx, hy, hz, u8[8][3], v8[8], th8[8], p8[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        gather_u8(P, ei, ej, ek, u, u8);
        gather_cell(P, ei, ej, ek, v, theta, thetaRef, p, v8, th8, p8);
        double D11[27], D22[27], D33[27], D12[27], D23[27], D13[27], ve[27], pe[27], te[27];
        double threekappa = 3. * m.lambda + 2. * m.mu, coefbeta = m.beta / threekappa;
        for (int g = 0; g < 27; g++)
          D11[g] = D22[g] = D33[g] = D12[g] = D23[g] = D13[g] = ve[g] = pe[g] = te[g] = 0.;
        for (int a = 0; a < 8; a++)
          for (int g = 0; g < 27; g++) {
            D11[g] += e.dphi[a][0][g] * u8[a][0];
            D22[g] += e.dphi[a][1][g] * u8[a][1];
            D33[g] += e.dphi[a][2][g] * u8[a][2];
            D12[g] += (e.dphi[a][0][g] * u8[a][1] + e.dphi[a][1][g] * u8[a][0]) * .5;
            D23[g] += (e.dphi[a][1][g] * u8[a][2] + e.dphi[a][2][g] * u8[a][1]) * .5;
            D13[g] += (e.dphi[a][0][g] * u8[a][2] + e.dphi[a][2][g] * u8[a][0]) * .5;
            ve[g] += e.phi[a][g] * v8[a];
            pe[g] += e.phi[a][g] * p8[a];
            te[g] += e.phi[a][g] * th8[a];
          }
        double El = 0.;
        for (int g = 0; g < 27; g++) {
          double tr = D11[g] + D22[g] + D33[g];
          D11[g] -= tr / 3.;
          D22[g] -= tr / 3.;
          D33[g] -= tr / 3.;
          El += (D11[g] * D11[g] + D22[g] * D22[g] + D33[g] * D33[g] +
                 (D12[g] * D12[g] + D23[g] * D23[g] + D13[g] * D13[g]) * 2.) *
                ve[g] * ve[g] * (1. + P->eta) * m.mu * e.w[g];
          /* NOCOMPRESSION (VF_ElasticEnergyNoCompression3D_local, VFMech.c:819-908): the
           * spherical factor is 1 instead of v where tr(eps) < 0 */
          const double sph = (P->unilateral && tr < 0.) ? 1. : ve[g];
          double WD = (tr / 3. - m.alpha * te[g]) * sph - coefbeta * pe[g];
          El += 3. * threekappa / 2. * WD * WD * e.w[g];
          El += threekappa / 6. * tr * tr * P->eta * e.w[g];
        }
        myE += El;
        if (P->hasCrackPressure) {
          double gv[3][27], ue[3][27], pe2[27];
          for (int g = 0; g < 27; g++) {
            pe2[g] = 0;
            for (int c = 0; c < 3; c++) gv[c][g] = ue[c][g] = 0.;
          }
          for (int a = 0; a < 8; a++)
            for (int g = 0; g < 27; g++) {
              pe2[g] += e.phi[a][g] * p8[a];
              for (int c = 0; c < 3; c++) {
                gv[c][g] += e.dphi[a][c][g] * v8[a];
                ue[c][g] += e.phi[a][g] * u8[a][c];
              }
            }
          for (int g = 0; g < 27; g++)
            myPW += e.w[g] * pe2[g] *
                    (ue[0][g] * gv[0][g] + ue[1][g] * gv[1][g] + ue[2][g] * gv[2][g]);
        }
      }
  out[0] = myE;
  out[1] = myPW;
  return 0;
}

/* VF_VEnergy3D (VFMech.c:2474-2526) with VF_AT1/AT2SurfaceEnergy3D_local
 * (VFMech.c:2394-2465). */
int vfo_v_energy(const vfo_problem *P, const double *v, double *surface) {
  double S = 0., hx, hy, hz, v8[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        cellmat m = cell_material(P, ei, ej, ek);
        gather_cell(P, ei, ej, ek, v, NULL, NULL, NULL, v8, NULL, NULL);
        double coef = m.Gc / atCv(P) * .25, ve[27], gv[3][27];
        for (int g = 0; g < 27; g++) ve[g] = gv[0][g] = gv[1][g] = gv[2][g] = 0.;
        for (int a = 0; a < 8; a++)
          for (int g = 0; g < 27; g++) {
            ve[g] += v8[a] * e.phi[a][g];
            gv[0][g] += v8[a] * e.dphi[a][0][g];
            gv[1][g] += v8[a] * e.dphi[a][1][g];
            gv[2][g] += v8[a] * e.dphi[a][2][g];
          }
        for (int g = 0; g < 27; g++) {
          double grad2 = gv[0][g] * gv[0][g] + gv[1][g] * gv[1][g] + gv[2][g] * gv[2][g];
          if (P->atnum == 1)
            S += e.w[g] * ((1. - ve[g]) / P->epsilon + grad2 * P->epsilon) * coef;
          else
            S += e.w[g] * ((1. - ve[g]) * (1. - ve[g]) / P->epsilon + grad2 * P->epsilon) * coef;
        }
      }
  *surface = S;
  return 0;
}

/* VolumetricCrackOpening (VFPermfield.c:15-152): COV = sum_e sum_g w (u . grad v). */
int vfo_cov(const vfo_problem *P, const double *u, const double *v, double *cov,
            double *cellcov) {
  double C = 0., hx, hy, hz, u8[8][3], v8[8];
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        gather_u8(P, ei, ej, ek, u, u8);
        gather_cell(P, ei, ej, ek, v, NULL, NULL, NULL, v8, NULL, NULL);
        double ud[3][27], dv[3][27];
        for (int g = 0; g < 27; g++)
          for (int c = 0; c < 3; c++) ud[c][g] = dv[c][g] = 0.;
        for (int g = 0; g < 27; g++)
          for (int a = 0; a < 8; a++)
            for (int c = 0; c < 3; c++) {
              ud[c][g] += u8[a][c] * e.phi[a][g];
              dv[c][g] += v8[a] * e.dphi[a][c][g];
            }
        double loc = 0., vol = 0., cell = 0.;
        for (int g = 0; g < 27; g++) {
          double t = (ud[0][g] * dv[0][g] + ud[1][g] * dv[1][g] + ud[2][g] * dv[2][g]) * e.w[g];
          cell += t;
          vol += e.w[g];
          loc += t;
        }
        if (cellcov) cellcov[((int64_t)ek * (P->ny - 1) + ej) * (P->nx - 1) + ei] = cell / vol;
        C += loc;
      }
  *cov = C;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Flow-coupling boundary: the fracture width UpdateFractureWidth
 * (VFPermfield.c:267-562) with CellToNodeInterpolation (VFPermfield.c:1156-1330), the
 * width integration length (VFCommon.c:897-914) and VolumetricFractureWellRate
 * (VFPermfield.c:1513-1604), restated serially in the reference's loop order. */

/* WidthIntLenght = 3 res + 4 epsilon, res the grid spacing picked by the reference's
 * comparison chain (VFCommon.c:897-914; for bx == by < bz it picks bz). */
double vfo_width_int_length(const vfo_problem *P) {
  const double bx = P->lx / (P->nx - 1), by = P->ly / (P->ny - 1), bz = P->lz / (P->nz - 1);
  double res;
  if (P->nx == 2) res = by < bz ? by : bz;
  else if (P->ny == 2) res = bx < bz ? bx : bz;
  else if (P->nz == 2) res = bx < by ? bx : by;
  else if (bx < by && bx < bz) res = bx;
  else if (by < bx && by < bz) res = by;
  else res = bz;
  return 3 * res + 4 * P->epsilon;
}

/* CartFEElement1DInit (VFCartFE.c:1773-1785): the linear basis at x in a segment of
 * length l, through the reference's map var = (x - l/2)/l/2 (so var stays in
 * [-1/4, 1/4] across the segment). */
static void pt_basis1d(double x, double l, double phi[2], double dphi[2]) {
  const double var = (x - l / 2.) / l / 2.;
  phi[0] = (1. - var) * .5;
  phi[1] = (1. + var) * .5;
  dphi[0] = -1. / l;
  dphi[1] = 1. / l;
}

typedef struct {
  double phi[8], dphi[8][3];
} ptelem;

/* CartFEElement3DInit (VFCartFE.c:1837-1866) at the point (x, y, z) of a cell. */
static void pt_elem(double x, double y, double z, double lx, double ly, double lz, ptelem *s) {
  double px[2], py[2], pz[2], dx[2], dy[2], dz[2];
  pt_basis1d(x, lx, px, dx);
  pt_basis1d(y, ly, py, dy);
  pt_basis1d(z, lz, pz, dz);
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) {
        const int a = i + 2 * j + 4 * k;
        s->phi[a] = pz[k] * py[j] * px[i];
        s->dphi[a][0] = pz[k] * py[j] * dx[i];
        s->dphi[a][1] = pz[k] * dy[j] * px[i];
        s->dphi[a][2] = dz[k] * py[j] * px[i];
      }
}

/* ComputeAveVGradVandNormal_local (VFPermfield.c:2124-2156): V, grad V, the unit
 * normal grad V / |grad V| (0 when not finite) and U at the point of cell (ei,ej,ek). */
static void pt_fields(const vfo_problem *P, const double *u, const double *v, int ei, int ej,
                      int ek, const ptelem *s, double *vave, double g[3], double n[3],
                      double uc[3]) {
  *vave = 0.;
  for (int c = 0; c < 3; c++) g[c] = n[c] = uc[c] = 0.;
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) {
        const int a = i + 2 * j + 4 * k;
        const int64_t q = NODE(P, ei + i, ej + j, ek + k);
        for (int c = 0; c < 3; c++) {
          g[c] += v[q] * s->dphi[a][c];
          uc[c] += u[3 * q + c] * s->phi[a];
        }
        *vave += v[q] * s->phi[a];
      }
  const double mag = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  for (int c = 0; c < 3; c++) n[c] = g[c] / mag;
  if (!isfinite(n[0]) || !isfinite(n[1]) || !isfinite(n[2])) n[0] = n[1] = n[2] = 0.;
}

/* IntegrateUcdotGradVlocal (VFPermfield.c:589-610) on the segment element of
 * VFCartFEElement1DInit(len): acc += sum_g (f0 phi_0 + f1 phi_1)(g) w_g / 2. */
static void seg_integrate(double *acc, double f0, double f1, const double w[3],
                          const double phi[2][3]) {
  double fe[3] = {0., 0., 0.};
  for (int i = 0; i < 2; i++)
    for (int g = 0; g < 3; g++) fe[g] += (i ? f1 : f0) * phi[i][g];
  for (int g = 0; g < 3; g++) *acc += fe[g] * w[g] / 2.;
}

/* The cell whose closed box holds coordinate c along one axis, the last one in the
 * reference's ascending scan (VFPermfield.c:370-384); -1 if none. */
static int axis_cell(double c, double l, int n) {
  for (int i = n - 2; i >= 0; i--)
    if (coord(i + 1, l, n) >= c && coord(i, l, n) <= c) return i;
  return -1;
}

/* One march of UpdateFractureWidth from the centre of cell (ei,ej,ek) along +n
 * (dir = 1, VFPermfield.c:356-440) or -n (dir = -1, :441-527); cur holds the cell
 * the previous point was found in (the reference keeps it when a point lies in no
 * cell).  Returns 0, or 1 if the march hit max_steps. */
static int width_march(const vfo_problem *P, const double *u, const double *v, int ei, int ej,
                       int ek, int dir, double len, double L, int cur[3], double *w,
                       double val[3], long max_steps) {
  double hx, hy, hz, vave, g[3], n[3], uc[3], ref[3], g0[3], ca[3], cc[3];
  ptelem s;
  cell_h(P, ei, ej, ek, &hx, &hy, &hz);
  pt_elem(hx / 2., hy / 2., hz / 2., hx, hy, hz, &s);
  pt_fields(P, u, v, ei, ej, ek, &s, &vave, g, n, uc);
  for (int c = 0; c < 3; c++) ref[c] = n[c];
  for (int c = 0; c < 3; c++) g0[c] = g[c];
  double cod0 = g[0] * uc[0] + g[1] * uc[1] + g[2] * uc[2];
  ca[0] = (coord(ei + 1, P->lx, P->nx) + coord(ei, P->lx, P->nx)) / 2.;
  ca[1] = (coord(ej + 1, P->ly, P->ny) + coord(ej, P->ly, P->ny)) / 2.;
  ca[2] = (coord(ek + 1, P->lz, P->nz) + coord(ek, P->lz, P->nz)) / 2.;
  for (int c = 0; c < 3; c++) cc[c] = dir > 0 ? ca[c] + n[c] * len : ca[c] - n[c] * len;
  double lc = len, sw[3], sphi[2][3], sdphi[2][3];
  tables1d(len, sw, sphi, sdphi); /* VFCartFEElement1DInit(len), VFCartFE.c:90-116 */
  long steps = 0;
  do {
    const int fi = axis_cell(cc[0], P->lx, P->nx), fj = axis_cell(cc[1], P->ly, P->ny),
              fk = axis_cell(cc[2], P->lz, P->nz);
    if (fi >= 0 && fj >= 0 && fk >= 0) {
      cur[0] = fi;
      cur[1] = fj;
      cur[2] = fk;
    }
    cell_h(P, cur[0], cur[1], cur[2], &hx, &hy, &hz);
    const double hwx = cc[0] - coord(cur[0], P->lx, P->nx);
    const double hwy = cc[1] - coord(cur[1], P->ly, P->ny);
    const double hwz = cc[2] - coord(cur[2], P->lz, P->nz);
    const double nold[3] = {n[0], n[1], n[2]};
    pt_elem(hwx, hwy, hwz, hx, hy, hz, &s);
    pt_fields(P, u, v, cur[0], cur[1], cur[2], &s, &vave, g, n, uc);
    const double cod1 = g[0] * uc[0] + g[1] * uc[1] + g[2] * uc[2];
    seg_integrate(w, cod0, cod1, sw, sphi);
    for (int c = 0; c < 3; c++) seg_integrate(&val[c], g0[c], g[c], sw, sphi);
    if (n[0] == 0 && n[1] == 0 && n[2] == 0)
      for (int c = 0; c < 3; c++) n[c] = nold[c];
    double c1[3], c2[3];
    for (int c = 0; c < 3; c++) {
      c1[c] = cc[c] + n[c] * len;
      c2[c] = cc[c] - n[c] * len;
    }
    const double t1 = sqrt((c1[0] - ca[0]) * (c1[0] - ca[0]) + (c1[1] - ca[1]) * (c1[1] - ca[1]) +
                           (c1[2] - ca[2]) * (c1[2] - ca[2]));
    const double t2 = sqrt((c2[0] - ca[0]) * (c2[0] - ca[0]) + (c2[1] - ca[1]) * (c2[1] - ca[1]) +
                           (c2[2] - ca[2]) * (c2[2] - ca[2]));
    if (t1 > t2) {
      for (int c = 0; c < 3; c++) cc[c] = c1[c];
    } else {
      for (int c = 0; c < 3; c++) {
        cc[c] = c2[c];
        n[c] = -1 * n[c];
      }
    }
    lc += len;
    cod0 = cod1;
    for (int c = 0; c < 3; c++) g0[c] = g[c];
    if (++steps >= max_steps) return 1;
  } while (lc < L - len && vave < 1.0 &&
           (dir > 0 ? ref[0] * n[0] + ref[1] * n[1] + ref[2] * n[2] >= 0.
                    : -ref[0] * n[0] - ref[1] * n[1] - ref[2] * n[2] >= 0.));
  return 0;
}

int vfo_fracture_width(const vfo_problem *P, const double *u, const double *v, double L,
                       double width_tol, int remove_tip, double *widthc, double *pmult,
                       int *nstall) {
  const long max_steps = 1000000;
  int cur[3] = {0, 0, 0}, stall = 0;
  double value = 0.; /* kept from cell to cell like the reference's */
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        const int64_t cell = ((int64_t)ek * (P->ny - 1) + ej) * (P->nx - 1) + ei;
        double hx, hy, hz, vave, g[3], n[3], uc[3], w = 0., val[3] = {0., 0., 0.};
        ptelem s;
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        pt_elem(hx / 2., hy / 2., hz / 2., hx, hy, hz, &s);
        pt_fields(P, u, v, ei, ej, ek, &s, &vave, g, n, uc);
        const double len =
            sqrt((n[0] * hx) * (n[0] * hx) + (n[1] * hy) * (n[1] * hy) + (n[2] * hz) * (n[2] * hz)) / 20;
        pmult[cell] = 1.;
        if (vave < 1.0 && vave > 0.0) {
          if (!(len > 0.)) {
            /* the reference's march does not advance here (and does not end) */
            stall++;
          } else {
            stall += width_march(P, u, v, ei, ej, ek, 1, len, L, cur, &w, val, max_steps);
            stall += width_march(P, u, v, ei, ej, ek, -1, len, L, cur, &w, val, max_steps);
            value = sqrt(val[0] * val[0] + val[1] * val[1] + val[2] * val[2]);
            if (value > width_tol) pmult[cell] = 0.;
          }
        }
        if (w < 0.0) w = 0;
        if (remove_tip && value > width_tol) w = 0;
        widthc[cell] = w;
      }
  if (nstall) *nstall = stall;
  return 0;
}

int vfo_cell_to_node(const vfo_problem *P, const double *cellv, double *nodev) {
  const int64_t N = (int64_t)P->nx * P->ny * P->nz;
  double *vol = (double *)calloc((size_t)N, sizeof(double));
  if (!vol) return -1;
  for (int64_t q = 0; q < N; q++) nodev[q] = 0.;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        const double c = cellv[((int64_t)ek * (P->ny - 1) + ej) * (P->nx - 1) + ei];
        double hx, hy, hz;
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        for (int k = 0; k < 2; k++)
          for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
              const int64_t q = NODE(P, ei + i, ej + j, ek + k);
              vol[q] += hz * hy * hx;
              nodev[q] += c * hx * hy * hz;
            }
      }
  for (int64_t q = 0; q < N; q++) nodev[q] = nodev[q] / vol[q];
  free(vol);
  return 0;
}

int vfo_fracture_well_rate(const vfo_problem *P, const double *v, const double *regrate,
                           double *rate) {
  double total = 0., hx, hy, hz;
  etab e;
  for (int ek = 0; ek < P->nz - 1; ek++)
    for (int ej = 0; ej < P->ny - 1; ej++)
      for (int ei = 0; ei < P->nx - 1; ei++) {
        cell_h(P, ei, ej, ek, &hx, &hy, &hz);
        etab_init(&e, hx, hy, hz);
        double dv[3][27], rg[27];
        for (int g = 0; g < 27; g++) {
          dv[0][g] = dv[1][g] = dv[2][g] = 0.;
          rg[g] = 0.;
        }
        for (int k = 0; k < 2; k++)
          for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
              const int a = i + 2 * j + 4 * k;
              const int64_t q = NODE(P, ei + i, ej + j, ek + k);
              for (int g = 0; g < 27; g++) {
                for (int c = 0; c < 3; c++) dv[c][g] += v[q] * e.dphi[a][c][g];
                rg[g] += regrate[q] * e.phi[a][g];
              }
            }
        double loc = 0.;
        for (int g = 0; g < 27; g++)
          loc += rg[g] * sqrt(dv[0][g] * dv[0][g] + dv[1][g] * dv[1][g] + dv[2][g] * dv[2][g]) * e.w[g];
        total += loc;
      }
  *rate = total;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* VFDistanceToPennyCrack (VFCracks.c:101-126) and VFPennyCrackBuildVAT1/2
 * (VFCracks.c:136-227). */
static double penny_distance(const double x[3], const double ctr[3], double r, double th,
                             double ph) {
  const double pi = 3.14159265358979323846264338327950288;
  double n[3], tau[3], l, xdotn;
  n[0] = cos(th * pi / 180.) * sin(ph * pi / 180.);
  n[1] = sin(th * pi / 180.) * sin(ph * pi / 180.);
  n[2] = cos(ph * pi / 180.);
  xdotn = (x[0] - ctr[0]) * n[0] + (x[1] - ctr[1]) * n[1] + (x[2] - ctr[2]) * n[2];
  tau[0] = (x[0] - ctr[0]) - xdotn * n[0];
  tau[1] = (x[1] - ctr[1]) - xdotn * n[1];
  tau[2] = (x[2] - ctr[2]) - xdotn * n[2];
  l = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
  if (l <= r) return sqrt(xdotn * xdotn);
  return sqrt(pow(xdotn, 2) + pow((l - r), 2));
}

int vfo_penny_crack_v(const vfo_problem *P, const double center[3], double r,
                      double theta_deg, double phi_deg, double thickness, double *v) {
  for (int k = 0; k < P->nz; k++)
    for (int j = 0; j < P->ny; j++)
      for (int i = 0; i < P->nx; i++) {
        double x[3] = {coord(i, P->lx, P->nx), coord(j, P->ly, P->ny), coord(k, P->lz, P->nz)};
        int64_t q = NODE(P, i, j, k);
        if (r == 0) {
          v[q] = 1.;
          continue;
        }
        double dist = penny_distance(x, center, r, theta_deg, phi_deg) - thickness / 2.;
        if (dist <= 0)
          v[q] = 0.;
        else if (P->atnum == 1)
          v[q] = dist < 2. * P->epsilon ? dist / P->epsilon * (1. - .25 * dist / P->epsilon) : 1.;
        else
          v[q] = 1. - exp(-dist / 2 / P->epsilon);
      }
  return 0;
}

/* VFDistanceToRectangularCrack (VFCracks.c:331-427): the crack is the parallelogram with
 * corners P1 = c[0..2], P2 = c[3..5], P3 = c[6..8] and P4 = 2C - P1, C = (P2 + P3)/2.
 * The in-plane distance from C to the edge along the direction of the projected point
 * is found from the angles the direction makes with C->P3 and C->P4; the operation
 * order (and the NaN that a point on the normal through C produces, which makes the
 * final test pick the plane distance) follows the reference. */
static void unit3(double a[3]) {
  double nn = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  a[0] = a[0] / nn;
  a[1] = a[1] / nn;
  a[2] = a[2] / nn;
}
static double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

double vfo_rect_distance(const double x[3], const double c[9]) {
  const double pi = 3.14159265358979323846264338327950288;
  double C[3], P4[3], a[3], b[3], n[3], tau[3], p[3], q[3], e1[3], e2[3], nq[3], side[3];
  for (int d = 0; d < 3; d++) {
    C[d] = (c[6 + d] + c[3 + d]) / 2.;
    P4[d] = 2. * C[d] - c[d];
    a[d] = c[3 + d] - c[d];
    b[d] = c[6 + d] - c[d];
  }
  n[0] = a[1] * b[2] - a[2] * b[1];
  n[1] = a[2] * b[0] - a[0] * b[2];
  n[2] = a[0] * b[1] - a[1] * b[0];
  unit3(n);
  double s = (x[0] - C[0]) * n[0] + (x[1] - C[1]) * n[1] + (x[2] - C[2]) * n[2];
  for (int d = 0; d < 3; d++) {
    tau[d] = (x[d] - C[d]) - s * n[d];
    p[d] = C[d] + s * n[d];
    q[d] = x[d] + C[d] - p[d];
    e1[d] = c[6 + d] - C[d];
    e2[d] = P4[d] - C[d];
  }
  unit3(e1);
  unit3(e2);
  const double theta_side = pi - acos(dot3(e2, e1));
  for (int d = 0; d < 3; d++) nq[d] = q[d] - C[d];
  unit3(nq);
  const double theta = acos(dot3(e2, nq)) + acos(-e1[0] * nq[0] - e1[1] * nq[1] - e1[2] * nq[2]);
  const int k = ((theta - theta_side) < 1e-6 || (2. * pi - theta_side - theta) < 1e-6) ? 3 : 6;
  for (int d = 0; d < 3; d++) side[d] = P4[d] - c[k + d];
  unit3(side);
  const double da = sqrt((P4[0] - C[0]) * (P4[0] - C[0]) + (P4[1] - C[1]) * (P4[1] - C[1]) +
                         (P4[2] - C[2]) * (P4[2] - C[2]));
  double db = fabs((P4[0] - C[0]) * side[0] + (P4[1] - C[1]) * side[1] + (P4[2] - C[2]) * side[2]);
  db = sqrt(da * da - db * db);
  const double to_side = db / sin(acos(dot3(side, nq)));
  const double l = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
  if (l > to_side) return sqrt((l - to_side) * (l - to_side) + s * s);
  return sqrt(s * s);
}

/* VFRectangularCrackBuildVAT1/AT2 (VFCracks.c:436-513).  AT1 subtracts half the
 * thickness from the distance; AT2 compares the raw distance with the full
 * thickness and uses it unshifted in the profile. */
int vfo_rect_crack_v(const vfo_problem *P, const double corners[9], double thickness,
                     double *v) {
  for (int k = 0; k < P->nz; k++)
    for (int j = 0; j < P->ny; j++)
      for (int i = 0; i < P->nx; i++) {
        double x[3] = {coord(i, P->lx, P->nx), coord(j, P->ly, P->ny), coord(k, P->lz, P->nz)};
        int64_t q = NODE(P, i, j, k);
        double dist = vfo_rect_distance(x, corners);
        if (P->atnum == 1) {
          dist -= thickness / 2.;
          if (dist <= 0)
            v[q] = 0.;
          else
            v[q] = dist < 2. * P->epsilon ? dist / P->epsilon * (1. - .25 * dist / P->epsilon) : 1.;
        } else {
          v[q] = dist <= thickness ? 0. : 1. - exp(-dist / 2 / P->epsilon);
        }
      }
  return 0;
}

/* VFFieldsInitialize (VFCommon.c:823-857): V = VIrrev = pointwise minimum over the
 * penny cracks (7 doubles each: center[3], r, theta, phi, thickness) and the
 * rectangular cracks (10 doubles each: corners[9], thickness), 1 where there is none. */
int vfo_cracks_v(const vfo_problem *P, int npenny, const double *penny, int nrect,
                 const double *rect, double *v) {
  const int64_t N = (int64_t)P->nx * P->ny * P->nz;
  double *w = (double *)malloc(N * sizeof(double));
  if (!w) return -1;
  for (int64_t q = 0; q < N; q++) v[q] = 1.;
  for (int c = 0; c < npenny + nrect; c++) {
    if (c < npenny) {
      const double *pc = penny + 7 * c;
      vfo_penny_crack_v(P, pc, pc[3], pc[4], pc[5], pc[6], w);
    } else {
      const double *rc = rect + 10 * (c - npenny);
      vfo_rect_crack_v(P, rc, rc[9], w);
    }
    for (int64_t q = 0; q < N; q++) v[q] = w[q] < v[q] ? w[q] : v[q];
  }
  free(w);
  return 0;
}
