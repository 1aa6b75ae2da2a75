// cracks.cu -- device crack initialisers: V = VIrrev = pointwise minimum over penny
// and rectangular cracks (VFFieldsInitialize, VFCommon.c:823-857).
//
// Everything that depends on the crack alone (normals, the rectangle's in-plane
// frame and side distances) is computed once on the host, with the operation order
// of the reference's per-point code; the kernel evaluates the per-node part.  This
// file is compiled without FMA contraction so that the arithmetic rounds like the
// reference's C code: the penny AT1 profile is reproduced bit for bit, while the
// AT2 exponential and the rectangle's acos/sin differ from the host libm by a few
// ulps at most.
#include <cmath>

#include "abi_util.h"

namespace vfgpu {
namespace {

constexpr int kBatch = 16;
constexpr double kPi = 3.14159265358979323846264338327950288;

struct PennyDev {
  double c[3], n[3], r, thickness;
  int zero;  // r == 0: the crack contributes v = 1
};

struct RectDev {
  double C[3], n[3], e1[3], e2[3], side[2][3], db[2];
  double theta_side, thickness;
};

struct CrackBatch {
  PennyDev p[kBatch];
  RectDev r[kBatch];
  int np, nr, first, atnum;
  int nx, ny, nz;
  double lx, ly, lz, eps;
};

void unit3(double a[3]) {
  const double nn = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  a[0] = a[0] / nn;
  a[1] = a[1] / nn;
  a[2] = a[2] / nn;
}

// VFDistanceToPennyCrack (VFCracks.c:101-126): the normal.
PennyDev penny_host(const vfgpu_penny& pc) {
  PennyDev d{};
  for (int k = 0; k < 3; k++) d.c[k] = pc.center[k];
  d.n[0] = std::cos(pc.theta * kPi / 180.) * std::sin(pc.phi * kPi / 180.);
  d.n[1] = std::sin(pc.theta * kPi / 180.) * std::sin(pc.phi * kPi / 180.);
  d.n[2] = std::cos(pc.phi * kPi / 180.);
  d.r = pc.r;
  d.thickness = pc.thickness;
  d.zero = pc.r == 0;
  return d;
}

// VFDistanceToRectangularCrack (VFCracks.c:331-427): center C, fourth corner
// P4 = 2C - P1, unit normal, unit directions C->P3 and C->P4, the angle between the
// sides, and for the two candidate sides (P4-P2, P4-P3) the unit direction and the
// distance from C to the side.
RectDev rect_host(const vfgpu_rect& rc) {
  const double* c = rc.corners;
  RectDev d{};
  double P4[3], a[3], b[3];
  for (int k = 0; k < 3; k++) {
    d.C[k] = (c[6 + k] + c[3 + k]) / 2.;
    P4[k] = 2. * d.C[k] - c[k];
    a[k] = c[3 + k] - c[k];
    b[k] = c[6 + k] - c[k];
  }
  d.n[0] = a[1] * b[2] - a[2] * b[1];
  d.n[1] = a[2] * b[0] - a[0] * b[2];
  d.n[2] = a[0] * b[1] - a[1] * b[0];
  unit3(d.n);
  for (int k = 0; k < 3; k++) {
    d.e1[k] = c[6 + k] - d.C[k];
    d.e2[k] = P4[k] - d.C[k];
  }
  unit3(d.e1);
  unit3(d.e2);
  d.theta_side = kPi - std::acos(d.e2[0] * d.e1[0] + d.e2[1] * d.e1[1] + d.e2[2] * d.e1[2]);
  const double da = std::sqrt((P4[0] - d.C[0]) * (P4[0] - d.C[0]) + (P4[1] - d.C[1]) * (P4[1] - d.C[1]) +
                              (P4[2] - d.C[2]) * (P4[2] - d.C[2]));
  for (int s = 0; s < 2; s++) {
    const int k0 = s == 0 ? 3 : 6;
    double* sd = d.side[s];
    for (int k = 0; k < 3; k++) sd[k] = P4[k] - c[k0 + k];
    unit3(sd);
    double db = std::fabs((P4[0] - d.C[0]) * sd[0] + (P4[1] - d.C[1]) * sd[1] + (P4[2] - d.C[2]) * sd[2]);
    d.db[s] = std::sqrt(da * da - db * db);
  }
  d.thickness = rc.thickness;
  return d;
}

__device__ double penny_v(const PennyDev& P, const double x[3], int atnum, double eps) {
  if (P.zero) return 1.;
  const double dx = x[0] - P.c[0], dy = x[1] - P.c[1], dz = x[2] - P.c[2];
  const double s = dx * P.n[0] + dy * P.n[1] + dz * P.n[2];
  const double t0 = dx - s * P.n[0], t1 = dy - s * P.n[1], t2 = dz - s * P.n[2];
  const double l = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
  double d = l <= P.r ? sqrt(s * s) : sqrt(s * s + (l - P.r) * (l - P.r));
  d -= P.thickness / 2.;
  if (d <= 0) return 0.;
  if (atnum == 1) return d < 2. * eps ? d / eps * (1. - .25 * d / eps) : 1.;
  return 1. - exp(-d / 2 / eps);
}

__device__ double rect_v(const RectDev& R, const double x[3], int atnum, double eps) {
  double tau[3], nq[3], s = 0;
  s = (x[0] - R.C[0]) * R.n[0] + (x[1] - R.C[1]) * R.n[1] + (x[2] - R.C[2]) * R.n[2];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    tau[k] = (x[k] - R.C[k]) - s * R.n[k];
    const double p = R.C[k] + s * R.n[k];
    const double q = x[k] + R.C[k] - p;
    nq[k] = q - R.C[k];
  }
  const double nn = sqrt(nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2]);
#pragma unroll
  for (int k = 0; k < 3; k++) nq[k] = nq[k] / nn;
  const double theta = acos(R.e2[0] * nq[0] + R.e2[1] * nq[1] + R.e2[2] * nq[2]) +
                       acos(-R.e1[0] * nq[0] - R.e1[1] * nq[1] - R.e1[2] * nq[2]);
  const int k = ((theta - R.theta_side) < 1e-6 || (2. * kPi - R.theta_side - theta) < 1e-6) ? 0 : 1;
  const double* sd = R.side[k];
  const double to_side = R.db[k] / sin(acos(sd[0] * nq[0] + sd[1] * nq[1] + sd[2] * nq[2]));
  const double l = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
  double d = l > to_side ? sqrt((l - to_side) * (l - to_side) + s * s) : sqrt(s * s);
  if (atnum == 1) {
    d -= R.thickness / 2.;
    if (d <= 0) return 0.;
    return d < 2. * eps ? d / eps * (1. - .25 * d / eps) : 1.;
  }
  return d <= R.thickness ? 0. : 1. - exp(-d / 2 / eps);
}

__device__ double node_coord(int i, double l, int n) { return i == 0 ? 0. : i * l / (n - 1.); }

__global__ void crack_kernel(const CrackBatch B, double* __restrict__ V, double* __restrict__ VI) {
  const int64_t N = (int64_t)B.nx * B.ny * B.nz;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % B.nx);
    const int j = (int)((q / B.nx) % B.ny);
    const int k = (int)(q / ((int64_t)B.nx * B.ny));
    const double x[3] = {node_coord(i, B.lx, B.nx), node_coord(j, B.ly, B.ny),
                         node_coord(k, B.lz, B.nz)};
    double v = B.first ? 1. : V[q];
    for (int c = 0; c < B.np; c++) v = fmin(v, penny_v(B.p[c], x, B.atnum, B.eps));
    for (int c = 0; c < B.nr; c++) v = fmin(v, rect_v(B.r[c], x, B.atnum, B.eps));
    V[q] = v;
    VI[q] = v;
  }
}

}  // namespace
}  // namespace vfgpu

using namespace vfgpu;

extern "C" int vfgpu_init_cracks(vfgpu_ctx* c, int npenny, const vfgpu_penny* penny, int nrect,
                                 const vfgpu_rect* rect) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_init_cracks: null ctx");
  if (npenny < 0 || nrect < 0 || (npenny && !penny) || (nrect && !rect))
    return fail(VFGPU_ERR_INVALID, "vfgpu_init_cracks: bad crack arrays");
  for (int q = 0; q < npenny; q++)
    if (!(penny[q].r >= 0) || !(penny[q].thickness >= 0))
      return fail(VFGPU_ERR_INVALID, "vfgpu_init_cracks: penny %d needs r >= 0, thickness >= 0", q);
  cudaSetDevice(c->dev);
  CrackBatch B{};
  B.atnum = c->vf.atnum;
  B.eps = c->vf.epsilon;
  B.nx = c->nx;
  B.ny = c->ny;
  B.nz = c->nz;
  B.lx = c->lx;
  B.ly = c->ly;
  B.lz = c->lz;
  const int blocks = (int)std::min<int64_t>((c->N + 255) / 256, (int64_t)c->nsm * 8);
  int ip = 0, ir = 0;
  B.first = 1;
  c->v32_stale = c->ul_stale = true;  // V changes from here on, also on an error return
  cudaError_t e = cudaSuccess;
  do {  // at least one pass, so that no cracks gives V = VIrrev = 1
    B.np = std::min(kBatch, npenny - ip);
    B.nr = std::min(kBatch, nrect - ir);
    for (int q = 0; q < B.np; q++) B.p[q] = penny_host(penny[ip + q]);
    for (int q = 0; q < B.nr; q++) B.r[q] = rect_host(rect[ir + q]);
    ip += B.np;
    ir += B.nr;
    crack_kernel<<<blocks, 256, 0, c->stream>>>(B, c->f[VFGPU_FIELD_V], c->f[VFGPU_FIELD_VIRREV]);
    e = cudaGetLastError();
    B.first = 0;
  } while (e == cudaSuccess && (ip < npenny || ir < nrect));
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_init_cracks");
  return VFGPU_OK;
}
