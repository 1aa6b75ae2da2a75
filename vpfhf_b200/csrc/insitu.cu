// insitu.cu -- in-situ boundary tractions: the load they add to the U residual
// (VF_GradientUInSituStresses3D_local, VFMech.c:598-715, applied in VF_UResidual,
// VFMech.c:1630-1848) and their work (VF_InSituStressWork3D_local, VFMech.c:983-1102,
// summed in VF_UEnergy3D, VFMech.c:1238-1407).
//
// On face F the traction is t_c = dir_F * s_comp(F,c)(z) with s linear in z between
// the stresses at z = 0 and z = lz; components with a Dirichlet BC on F get none.
// The reference spreads a face cell's load over the whole boundary element and then
// adds every row to the face layer, so each face node receives the consistent surface
// load int_face phi_node t dA of the bilinearly interpolated traction; here that
// integral is evaluated exactly (bilinear x bilinear: the 1-D mass matrix
// h/6 [2 1; 1 2] per in-plane axis).  The work follows VF_UEnergy3D, which takes the
// X1/Y1/Z1 faces at cell index (cells - 2), i.e. at the node layer one inside the box
// (none when that axis has a single cell), and integrates u . t over each face cell.
// Deterministic: gathers per node in a fixed order, fixed-order block reductions.
#include <algorithm>

#include "elem.h"

namespace vfgpu {
namespace {

// stress component (Voigt) of each traction component, and the sign of the normal
__device__ __forceinline__ int comp_of(int face, int c) {
  const int t[6][3] = {{0, 5, 4}, {0, 5, 4}, {5, 1, 3}, {5, 1, 3}, {4, 3, 2}, {4, 3, 2}};
  return t[face][c];
}
__device__ __forceinline__ double traction(const InsituArgs& A, int face, int c, double z) {
  const int s = comp_of(face, c);
  const double dir = (face & 1) ? 1. : -1.;
  return dir * (A.smin[s] + (z - 0.) / (A.lz - 0.) * (A.smax[s] - A.smin[s]));
}
__device__ __forceinline__ double zcoord(const InsituArgs& A, int k) {
  return k == 0 ? 0. : k * A.lz / (A.nz - 1.);
}

// Face geometry: in-plane node counts (na, nb), spacings, and the node of in-plane
// index (a, b) on node layer `layer` of the face's normal axis.  X faces: (a, b) =
// (j, k); Y faces: (i, k); Z faces: (i, j).
struct FaceGeo {
  int na, nb;
  double ha, hb;
};
__device__ __forceinline__ FaceGeo face_geo(const InsituArgs& A, int face) {
  if (face < 2) return {A.ny, A.nz, A.hy, A.hz};
  if (face < 4) return {A.nx, A.nz, A.hx, A.hz};
  return {A.nx, A.ny, A.hx, A.hy};
}
__device__ __forceinline__ int64_t face_node(const InsituArgs& A, int face, int layer, int a, int b) {
  if (face < 2) return node_index(layer, a, b, A.nx, A.ny);
  if (face < 4) return node_index(a, layer, b, A.nx, A.ny);
  return node_index(a, b, layer, A.nx, A.ny);
}
// z of in-plane node (a, b) of a face on node layer `layer`
__device__ __forceinline__ double face_z(const InsituArgs& A, int face, int layer, int b) {
  return face < 4 ? zcoord(A, b) : zcoord(A, layer);
}

__global__ void insitu_load_kernel(const InsituArgs A, int face, double* __restrict__ f) {
  const FaceGeo G = face_geo(A, face);
  const int layer = (face & 1) ? (face < 2 ? A.nx - 1 : face < 4 ? A.ny - 1 : A.nz - 1) : 0;
  const int64_t nn = (int64_t)G.na * G.nb;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nn;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(t % G.na), b = (int)(t / G.na);
    double load[3] = {0., 0., 0.};
    // the (up to) four face cells around the node, in a fixed order
#pragma unroll
    for (int db = -1; db <= 0; db++)
#pragma unroll
      for (int da = -1; da <= 0; da++) {
        const int ca = a + da, cb = b + db;
        if (ca < 0 || cb < 0 || ca >= G.na - 1 || cb >= G.nb - 1) continue;
        const int ia = -da, ib = -db;  // the node's corner in the cell
#pragma unroll
        for (int c = 0; c < 3; c++) {
          if (!A.freec[face][c]) continue;
          double s = 0.;
#pragma unroll
          for (int q = 0; q < 2; q++)
#pragma unroll
            for (int p = 0; p < 2; p++) {
              const double tv = traction(A, face, c, face_z(A, face, layer, cb + q));
              s += (p == ia ? 2. : 1.) * (q == ib ? 2. : 1.) * tv;
            }
          load[c] += s * (G.ha * G.hb / 36.);
        }
      }
    const int64_t n = face_node(A, face, layer, a, b);
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (A.freec[face][c]) f[3 * n + c] += load[c];
  }
}

constexpr int W_BLOCKS = 64, W_THREADS = 256;

__global__ void __launch_bounds__(W_THREADS) insitu_work_kernel(const InsituArgs A,
                                                                 const double* __restrict__ u,
                                                                 double* __restrict__ partial) {
  __shared__ double red[32];
  const int face = blockIdx.y;
  const FaceGeo G = face_geo(A, face);
  const int n1 = face < 2 ? A.nx : face < 4 ? A.ny : A.nz;
  // VF_UEnergy3D: "0" faces at the first cell, "1" faces at cell (cells - 2), whose far
  // node layer is n1 - 2
  const int layer = (face & 1) ? n1 - 2 : 0;
  const bool on = !(face & 1) || n1 >= 3;
  const int64_t ncell = on ? (int64_t)(G.na - 1) * (G.nb - 1) : 0;
  double w = 0.;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ncell;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int ca = (int)(t % (G.na - 1)), cb = (int)(t / (G.na - 1));
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (!A.freec[face][c]) continue;
      double s = 0.;
#pragma unroll
      for (int q = 0; q < 2; q++)
#pragma unroll
        for (int p = 0; p < 2; p++) {
          const double uv = u[3 * face_node(A, face, layer, ca + p, cb + q) + c];
          double mt = 0.;  // sum over the cell's nodes of the mass weights times t
#pragma unroll
          for (int q2 = 0; q2 < 2; q2++)
#pragma unroll
            for (int p2 = 0; p2 < 2; p2++)
              mt += (p == p2 ? 2. : 1.) * (q == q2 ? 2. : 1.) *
                    traction(A, face, c, face_z(A, face, layer, cb + q2));
          s += uv * mt;
        }
      w += s * (G.ha * G.hb / 36.);
    }
  }
  const double bs = block_sum_dbl(w, red);
  if (threadIdx.x == 0) partial[face * W_BLOCKS + blockIdx.x] = bs;
}

__global__ void insitu_work_final(const double* __restrict__ partial, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double s = 0.;
  for (int b = 0; b < 6 * W_BLOCKS; b++) s += partial[b];
  out[0] = s;
}

}  // namespace

cudaError_t launch_insitu_load(const InsituArgs& A, double* f, cudaStream_t s) {
  for (int face = 0; face < 6; face++) {
    if (!(A.freec[face][0] || A.freec[face][1] || A.freec[face][2])) continue;
    const int64_t nn = face < 2 ? (int64_t)A.ny * A.nz : face < 4 ? (int64_t)A.nx * A.nz
                                                                  : (int64_t)A.nx * A.ny;
    const int blocks = (int)std::min<int64_t>((nn + 255) / 256, 148 * 4);
    insitu_load_kernel<<<blocks, 256, 0, s>>>(A, face, f);
  }
  return cudaGetLastError();
}

cudaError_t launch_insitu_work(const InsituArgs& A, const double* u, double* partial, double* out,
                               cudaStream_t s) {
  insitu_work_kernel<<<dim3(W_BLOCKS, 6), W_THREADS, 0, s>>>(A, u, partial);
  insitu_work_final<<<1, 32, 0, s>>>(partial, out);
  return cudaGetLastError();
}

}  // namespace vfgpu
