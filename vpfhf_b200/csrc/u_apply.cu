// u_apply.cu -- kernels and launcher for the matrix-free U operator.
#include "kernels.h"
#include "u_apply.cuh"

namespace vfgpu {

template <typename T, int TY>
__global__ void __launch_bounds__(32 * TY, sizeof(T) == 8 ? 1 : 2)
    u_apply_kernel(const UApplyArgs<T> A, const LayerTable L) {
  using G = UTile<TY>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sx = reinterpret_cast<T*>(smem_raw);  // [2 buf][4 comp][BY][BX]: u0,u1,u2,v
  T* sc = sx + 2 * 4 * G::BY * G::BX;      // [24 = corner*3+c][TY][32]
  const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
  const int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
  const int X0 = bx * 32, Y0 = by * TY;
  const int nx = A.nx, ny = A.ny, nz = A.nz, nex = nx - 1, ney = ny - 1;
  const int z0 = bz * A.zc;
  if (z0 >= nz) return;
  const int z1 = min(z0 + A.zc, nz);
  const int kf = max(z0 - 1, 0), kl = min(z1, nz - 1) - 1;

#define SXA(buf, comp, w, l) sx[(((buf) * 4 + (comp)) * G::BY + (w)) * G::BX + (l)]
#define SCA(q, w, l) sc[((q) * TY + (w)) * 32 + (l)]

  auto load_plane = [&](int buf, int kz) {
    for (int s = tid; s < G::BX * G::BY; s += G::NT) {
      const int l = s % G::BX, w = s / G::BX, X = X0 + l, Y = Y0 + w;
      T u0 = T(0), u1 = T(0), u2 = T(0), vv = T(0);
      if (X < nx && Y < ny) {
        const int64_t n = node_index(X, Y, kz, nx, ny);
        u0 = A.x[3 * n];
        u1 = A.x[3 * n + 1];
        u2 = A.x[3 * n + 2];
        vv = A.v[n];
      }
      SXA(buf, 0, w, l) = u0;
      SXA(buf, 1, w, l) = u1;
      SXA(buf, 2, w, l) = u2;
      SXA(buf, 3, w, l) = vv;
    }
  };

  auto emit = [&](int l, int w, int X, int Y, int z, const T (&val)[3]) {
    const bool left = (l == 0 && bx > 0), right = (l == 32 && bx < A.ntx - 1);
    const bool bot = (w == 0 && by > 0), top = (w == TY && by < A.nty - 1);
    const int64_t n = node_index(X, Y, z, nx, ny);
    if (!(left || right || bot || top)) {
      const unsigned b = A.bc ? A.bc[n] : 0u;
#pragma unroll
      for (int c = 0; c < 3; c++) A.y[3 * n + c] = ((b >> c) & 1u) ? A.x[3 * n + c] : val[c];
    } else if (left || right) {
      const int i = left ? bx : bx + 1;
      const int slot = (bot ? 2 : 0) + (left ? 1 : 0);
      T* p = A.seamX + ((((int64_t)(i - 1) * nz + z) * ny + Y) * 4 + slot) * 3;
#pragma unroll
      for (int c = 0; c < 3; c++) p[c] = val[c];
    } else {
      const int j = bot ? by : by + 1;
      T* p = A.seamY + ((((int64_t)(j - 1) * nz + z) * nx + X) * 2 + (bot ? 1 : 0)) * 3;
#pragma unroll
      for (int c = 0; c < 3; c++) p[c] = val[c];
    }
  };

  T carry[G::NSLOT][3];
#pragma unroll
  for (int si = 0; si < G::NSLOT; si++)
#pragma unroll
    for (int c = 0; c < 3; c++) carry[si][c] = T(0);

  load_plane(0, kf);
  int cur = 0;
  for (int k = kf; k <= kl; k++) {
    load_plane(cur ^ 1, k + 1);
    __syncthreads();
    const int ex = X0 + lane, ey = Y0 + wy;
    T yc[8][3];
    if (ex < nex && ey < ney) {
      T xn[8][3], vn[8];
#pragma unroll
      for (int kk = 0; kk < 2; kk++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
          for (int i = 0; i < 2; i++) {
            const int a = i + 2 * j + 4 * kk, buf = kk ? cur ^ 1 : cur;
#pragma unroll
            for (int c = 0; c < 3; c++) xn[a][c] = SXA(buf, c, wy + j, lane + i);
            vn[a] = SXA(buf, 3, wy + j, lane + i);
          }
      const int layer = A.elayer ? A.elayer[k] : 0;
      T lam, mu;
      if (A.cellE) {
        const T E = T(A.cellE[((int64_t)k * ney + ey) * nex + ex]);
        lam = E * T(L.lamfac[layer]);
        mu = E * T(L.mufac[layer]);
      } else {
        lam = T(L.lambda[layer]);
        mu = T(L.mu[layer]);
      }
      u_element<T>(xn, vn, lam, mu, A.eta, A.ihx, A.ihy, A.ihz, A.vol, yc);
    } else {
#pragma unroll
      for (int a = 0; a < 8; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) yc[a][c] = T(0);
    }
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int c = 0; c < 3; c++) SCA(a * 3 + c, wy, lane) = yc[a][c];
    __syncthreads();
#pragma unroll
    for (int si = 0; si < G::NSLOT; si++) {
      const int s = tid + si * G::NT;
      if (s >= G::BX * G::BY) continue;
      const int l = s % G::BX, w = s / G::BX, X = X0 + l, Y = Y0 + w;
      if (X >= nx || Y >= ny) continue;
      T p0[3] = {T(0), T(0), T(0)}, p1[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int dw = 0; dw < 2; dw++) {
        const int ew = w - 1 + dw, j = 1 - dw;
        if (ew < 0 || ew >= TY) continue;
#pragma unroll
        for (int dl = 0; dl < 2; dl++) {
          const int el = l - 1 + dl, i = 1 - dl;
          if (el < 0 || el >= 32) continue;
#pragma unroll
          for (int c = 0; c < 3; c++) {
            p0[c] += SCA((i + 2 * j) * 3 + c, ew, el);
            p1[c] += SCA((i + 2 * j + 4) * 3 + c, ew, el);
          }
        }
      }
      if (k >= z0) {
        T val[3];
#pragma unroll
        for (int c = 0; c < 3; c++) val[c] = carry[si][c] + p0[c];
        emit(l, w, X, Y, k, val);
      }
#pragma unroll
      for (int c = 0; c < 3; c++) carry[si][c] = p1[c];
    }
    cur ^= 1;
  }
  if (z1 == nz) {
#pragma unroll
    for (int si = 0; si < G::NSLOT; si++) {
      const int s = tid + si * G::NT;
      if (s >= G::BX * G::BY) continue;
      const int l = s % G::BX, w = s / G::BX, X = X0 + l, Y = Y0 + w;
      if (X >= nx || Y >= ny) continue;
      emit(l, w, X, Y, nz - 1, carry[si]);
    }
  }
#undef SXA
#undef SCA
}

// Sums the 2 (or 4, where an x-seam crosses a y-seam) tile partials of every seam
// node in a fixed order and applies the Dirichlet rows.
template <typename T>
__global__ void u_seam_fixup_kernel(const UApplyArgs<T> A, int TY) {
  const int nx = A.nx, ny = A.ny, nz = A.nz;
  const int64_t nxs = (int64_t)(A.ntx - 1) * nz * ny;
  const int64_t nys = (int64_t)(A.nty - 1) * nz * nx;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nxs + nys;
       t += (int64_t)gridDim.x * blockDim.x) {
    T val[3];
    int64_t n;
    if (t < nxs) {
      const int Y = (int)(t % ny);
      const int64_t r = t / ny;
      const int z = (int)(r % nz), i = (int)(r / nz) + 1;
      const bool onY = (Y % TY == 0) && (Y > 0) && (Y / TY < A.nty);
      const T* p = A.seamX + t * 12;
#pragma unroll
      for (int c = 0; c < 3; c++)
        val[c] = onY ? ((p[c] + p[3 + c]) + p[6 + c]) + p[9 + c] : p[c] + p[3 + c];
      n = node_index(32 * i, Y, z, nx, ny);
    } else {
      const int64_t u = t - nxs;
      const int X = (int)(u % nx);
      const int64_t r = u / nx;
      const int z = (int)(r % nz), j = (int)(r / nz) + 1;
      if (X % 32 == 0 && X > 0 && X / 32 < A.ntx) continue;
      const T* p = A.seamY + u * 6;
#pragma unroll
      for (int c = 0; c < 3; c++) val[c] = p[c] + p[3 + c];
      n = node_index(X, TY * j, z, nx, ny);
    }
    const unsigned b = A.bc ? A.bc[n] : 0u;
#pragma unroll
    for (int c = 0; c < 3; c++) A.y[3 * n + c] = ((b >> c) & 1u) ? A.x[3 * n + c] : val[c];
  }
}

constexpr int U_TY = 8;

UPlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms) {
  UPlan p;
  p.ty = U_TY;
  p.ntx = ceil_div(nx - 1, 32);
  p.nty = ceil_div(ny - 1, U_TY);
  const int per_sm = prec_bytes == 8 ? 1 : 2;
  const int slots = num_sms * per_sm, tiles = p.ntx * p.nty;
  double best = 1e300;
  p.zc = nz;
  for (int nzc = 1; nzc <= nz; nzc++) {
    const int zc = ceil_div(nz, nzc), chunks = ceil_div(nz, zc);
    const int waves = ceil_div(tiles * chunks, slots);
    const double cost = (double)waves * (zc + 1 + 2);  // +1 halo layer, +2 fill/drain
    if (cost < best - 1e-9) {
      best = cost;
      p.zc = zc;
    }
  }
  p.nzc = ceil_div(nz, p.zc);
  p.seamX = (size_t)(p.ntx - 1) * nz * ny * 12;
  p.seamY = (size_t)(p.nty - 1) * nz * nx * 6;
  return p;
}

template <typename T>
cudaError_t launch_u_apply(const UApplyArgs<T>& A0, const UPlan& p, const LayerTable& L,
                           cudaStream_t s) {
  UApplyArgs<T> A = A0;
  A.ntx = p.ntx;
  A.nty = p.nty;
  A.zc = p.zc;
  const size_t smem = u_apply_smem_bytes<T, U_TY>();
  static bool attr_set = false;  // per template instance
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(u_apply_kernel<T, U_TY>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  dim3 grid(p.ntx, p.nty, p.nzc), block(32, U_TY);
  u_apply_kernel<T, U_TY><<<grid, block, smem, s>>>(A, L);
  const int64_t nseam = (int64_t)(p.ntx - 1) * A.nz * A.ny + (int64_t)(p.nty - 1) * A.nz * A.nx;
  if (nseam > 0) {
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>((nseam + threads - 1) / threads, 148 * 8);
    u_seam_fixup_kernel<T><<<blocks, threads, 0, s>>>(A, U_TY);
  }
  return cudaGetLastError();
}

template cudaError_t launch_u_apply<double>(const UApplyArgs<double>&, const UPlan&,
                                            const LayerTable&, cudaStream_t);
template cudaError_t launch_u_apply<float>(const UApplyArgs<float>&, const UPlan&,
                                           const LayerTable&, cudaStream_t);

}  // namespace vfgpu
