// tc_apply.cu -- the degraded elasticity operator y = K(v) x with its element
// contraction on the 5th-generation tensor cores (tcgen05.mma, accumulators in
// tensor memory), FP32 data, split-TF32 products (hi/lo, three products per term).
//
// A measured alternative to the CUDA-core modal element (u_apply.cuh), kept beside
// it and not used by the solvers.  Written as two GEMMs over the elements of a tile
// (VF_BilinearFormU3D_local, VFMech.c:227-290, applied as in VF_UResidual,
// VFMech.c:1555-1596):
//   GEMM1  D1[e][8 g + q] = sum_k A1[e][k] B1[k][8 g + q]   (M = 128 elements, K = 32,
//          N = 224): A1 = the element's 24 nodal displacements and 8 nodal phase-field
//          values; per Gauss point g the columns give tr(grad u), the engineering strain
//          with doubled normal components (2 e_xx, 2 e_yy, 2 e_zz, g_xy, g_xz, g_yz) and
//          v(g);
//   pointwise (CUDA cores): s = v(g)^2 + eta, then lambda s tr and mu s E_q -- 7 values
//          per point, 189 per element;
//   GEMM2  y[e][3 a + c] = sum_k A2[e][k] B2[k][3 a + c] (K = 189 padded to 192 in three
//          passes of 9 points x 7 + 1 zero column, N = 32 with 24 used), B2 holding the
//          Gauss-weighted divergence and strain of the test functions.
// Split TF32: every FP32 operand x is hi + lo with hi = tf32(x), lo = tf32(x - hi); a
// product is hi hi + hi lo + lo hi (the lo lo term, ~2^-22 relative, is dropped), so
// each GEMM is three MMAs per K step, accumulated in FP32 in tensor memory.
//
// Schedule: a persistent CTA of 128 threads (4 warps) per SM walks tiles of
// 32 x 4 elements of one element layer; thread m owns tile row m = TMEM lane m.
// Shared memory holds B1, B2 (hi and lo, loaded once), A1 and one third of A2 (hi and
// lo), all in the K-major no-swizzle canonical layout (8-row x 16-byte core matrices):
// 200 KB, one CTA per SM; tensor memory 256 columns (D1: 0..223, D2: 224..255).
// Element results are added into y with atomics; Dirichlet rows are set to x by a
// second kernel.  Every mbarrier wait is bounded: a block whose wait gives up flags
// A.err, stops issuing work, waits (bounded) for the MMAs it issued and frees its
// tensor memory before returning.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "abi_util.h"
#include "kernels.h"

namespace vfgpu {
namespace {

constexpr int TC_M = 128;      // elements per tile (MMA M)
constexpr int TC_TY = 4;       // tile rows: 32 x 4 elements
constexpr int TC_K1 = 32;      // GEMM1 K: 24 displacements + 8 phase-field values
constexpr int TC_N1 = 224;     // GEMM1 N: 27 points x 8 columns + 8 zero columns
constexpr int TC_KP = 64;      // GEMM2 K per pass: 9 points x 7 + 1 zero column
constexpr int TC_K2 = 3 * TC_KP;
constexpr int TC_N2 = 32;      // GEMM2 N: 24 dofs + 8 zero columns
constexpr int TC_TMEM_COLS = 256;
constexpr int TC_D2_COL = TC_N1;

// Byte offset of element (r, k) of an R-row operand in the K-major no-swizzle
// canonical layout: core matrices of 8 rows x 16 bytes (4 FP32/TF32 values), the
// 8-row groups 128 bytes apart (SBO), the 4-value K chunks R x 16 bytes apart (LBO).
__host__ __device__ constexpr uint32_t canon(int R, int r, int k) {
  return (uint32_t)((k >> 2) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// Shared-memory map (bytes)
constexpr uint32_t SZ_B1 = TC_N1 * TC_K1 * 4;   // 28672
constexpr uint32_t SZ_B2 = TC_N2 * TC_K2 * 4;   // 24576
constexpr uint32_t SZ_A1 = TC_M * TC_K1 * 4;    // 16384
constexpr uint32_t SZ_A2 = TC_M * TC_KP * 4;    // 32768
constexpr uint32_t OFF_B1H = 0, OFF_B1L = OFF_B1H + SZ_B1;
constexpr uint32_t OFF_B2H = OFF_B1L + SZ_B1, OFF_B2L = OFF_B2H + SZ_B2;
constexpr uint32_t OFF_A1H = OFF_B2L + SZ_B2, OFF_A1L = OFF_A1H + SZ_A1;
constexpr uint32_t OFF_A2H = OFF_A1L + SZ_A1, OFF_A2L = OFF_A2H + SZ_A2;
constexpr uint32_t OFF_BAR = OFF_A2L + SZ_A2;   // 2 mbarriers
constexpr uint32_t OFF_TMEM = OFF_BAR + 16;     // tensor-memory address from tcgen05.alloc
constexpr uint32_t TC_SMEM = OFF_TMEM + 16;
static_assert(TC_SMEM <= 227 * 1024, "shared memory of the tensor-core apply");

struct TcArgs {
  const float* __restrict__ x;      // 3N
  const float* __restrict__ v;      // N
  float* __restrict__ y;            // 3N, zeroed before the launch
  const uint32_t* __restrict__ B;   // B1 hi, B1 lo, B2 hi, B2 lo in the canonical layouts
  const uint8_t* __restrict__ elayer;
  const float* __restrict__ cellE;
  const DevParams* __restrict__ P;
  unsigned* __restrict__ err;       // set when a bounded wait gives up
  int nx, ny, nz, ntx, nty;
  long long ntiles;
};

// ---- tcgen05 / mbarrier primitives --------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t to_tf32(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return r;
}

// Smem matrix descriptor: start address, LBO and SBO in 16-byte units, version 1,
// no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32, FP32 accumulate, A and B K-major, M = 128.
constexpr uint32_t idesc_tf32(int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t addr, float (&r)[8]) {
  uint32_t u[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]),
                 "=r"(u[7])
               : "r"(addr));
#pragma unroll
  for (int i = 0; i < 8; i++) r[i] = __uint_as_float(u[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void bar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
// Bounded parity wait (~1 s at the top clock); false if it gave up.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 2000000000ll) return false;
  }
}

// Splits a into TF32 hi/lo and stores both at byte offset off of the two buffers.
__device__ __forceinline__ void put_split(unsigned char* sm, uint32_t off_hi, uint32_t off_lo, uint32_t o,
                                          float a) {
  const uint32_t h = to_tf32(a);
  const uint32_t l = to_tf32(a - __uint_as_float(h));
  *reinterpret_cast<uint32_t*>(sm + off_hi + o) = h;
  *reinterpret_cast<uint32_t*>(sm + off_lo + o) = l;
}

__global__ void __launch_bounds__(128, 1) tc_u_apply_kernel(const TcArgs A) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = smem_u32(sm);
  const uint32_t bar1 = sbase + OFF_BAR, bar2 = sbase + OFF_BAR + 8;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + OFF_TMEM);

  // constant operands B1, B2 (hi and lo), already in the canonical layouts
  {
    const uint4* src = reinterpret_cast<const uint4*>(A.B);
    uint4* dst = reinterpret_cast<uint4*>(sm);
    for (uint32_t i = tid; i < (2 * SZ_B1 + 2 * SZ_B2) / 16; i += blockDim.x) dst[i] = src[i];
    // the zero pad column k = 63 of every A2 pass; never written afterwards
    for (int r = tid; r < TC_M; r += blockDim.x) {
      *reinterpret_cast<uint32_t*>(sm + OFF_A2H + canon(TC_M, r, TC_KP - 1)) = 0u;
      *reinterpret_cast<uint32_t*>(sm + OFF_A2L + canon(TC_M, r, TC_KP - 1)) = 0u;
    }
  }
  if (tid == 0) {
    bar_init(bar1);
    bar_init(bar2);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;

  const int nx = A.nx, ny = A.ny, nex = nx - 1, ney = ny - 1;
  const LayerTable& LT = A.P->L;
  const float eta = (float)A.P->eta;
  constexpr uint32_t ID1 = idesc_tf32(TC_N1), ID2 = idesc_tf32(TC_N2);
  uint32_t ph1 = 0, ph2 = 0;  // completed phases of bar1 / bar2
  bool ok = true;
  int issued1 = 0, issued2 = 0;  // commits not yet waited for (for the clean-up)

  for (long long t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const int per_layer = A.ntx * A.nty;
    const int ez = (int)(t / per_layer), rem = (int)(t % per_layer);
    const int bx = rem % A.ntx, by = rem / A.ntx;
    const int ex = 32 * bx + lane, ey = TC_TY * by + warp;
    const bool valid = ex < nex && ey < ney;
    int64_t node[8];
#pragma unroll
    for (int a = 0; a < 8; a++)
      node[a] = ((int64_t)(ez + (a >> 2)) * ny + (ey + ((a >> 1) & 1))) * nx + ex + (a & 1);
    // ---- A1 row: displacements (k = 3 a + c) and phase field (k = 24 + a)
#pragma unroll
    for (int a = 0; a < 8; a++) {
#pragma unroll
      for (int c = 0; c < 3; c++)
        put_split(sm, OFF_A1H, OFF_A1L, canon(TC_M, tid, 3 * a + c), valid ? A.x[3 * node[a] + c] : 0.f);
      put_split(sm, OFF_A1H, OFF_A1L, canon(TC_M, tid, 24 + a), valid ? A.v[node[a]] : 0.f);
    }
    float lam = 0.f, mu = 0.f;
    if (valid) {
      const int layer = A.elayer ? A.elayer[ez] : 0;
      if (A.cellE) {
        const float E = A.cellE[((int64_t)ez * ney + ey) * nex + ex];
        lam = E * (float)LT.lamfac[layer];
        mu = E * (float)LT.mufac[layer];
      } else {
        lam = (float)LT.lambda[layer];
        mu = (float)LT.mu[layer];
      }
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    // ---- GEMM1 (one thread issues): D1 = A1h B1h + A1h B1l + A1l B1h
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < TC_K1 / 8; s++) {
        const uint32_t ka = (uint32_t)(2 * s) * (TC_M * 16), kb = (uint32_t)(2 * s) * (TC_N1 * 16);
        const uint64_t a_h = sdesc(sbase + OFF_A1H + ka, TC_M * 16, 128);
        const uint64_t a_l = sdesc(sbase + OFF_A1L + ka, TC_M * 16, 128);
        const uint64_t b_h = sdesc(sbase + OFF_B1H + kb, TC_N1 * 16, 128);
        const uint64_t b_l = sdesc(sbase + OFF_B1L + kb, TC_N1 * 16, 128);
        mma_tf32(tmem, a_h, b_h, ID1, s > 0);
        mma_tf32(tmem, a_h, b_l, ID1, 1);
        mma_tf32(tmem, a_l, b_h, ID1, 1);
      }
      mma_commit(bar1);
    }
    issued1++;
    if (__syncthreads_or(!bar_wait(bar1, ph1 & 1))) {
      ok = false;
      break;
    }
    ph1++;
    issued1--;
    tc_fence_after();
    // ---- three passes of 9 Gauss points: pointwise stress -> A2 -> GEMM2
    for (int pass = 0; pass < 3 && ok; pass++) {
      if (pass > 0) {  // the previous pass's MMAs still read A2
        if (__syncthreads_or(!bar_wait(bar2, ph2 & 1))) {
          ok = false;
          break;
        }
        ph2++;
        issued2--;
      }
#pragma unroll
      for (int i = 0; i < 9; i++) {
        const int g = 9 * pass + i;
        float r[8];
        tmem_ld8(tmem + lane_base + 8 * g, r);
        tmem_wait_ld();
        const float s = fmaf(r[7], r[7], eta);
        const float ls = lam * s, ms = mu * s;
        put_split(sm, OFF_A2H, OFF_A2L, canon(TC_M, tid, 7 * i), ls * r[0]);
#pragma unroll
        for (int q = 1; q < 7; q++) put_split(sm, OFF_A2H, OFF_A2L, canon(TC_M, tid, 7 * i + q), ms * r[q]);
      }
      proxy_fence();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < TC_KP / 8; s++) {
          const uint32_t ka = (uint32_t)(2 * s) * (TC_M * 16);
          const uint32_t kb = (uint32_t)(2 * (8 * pass + s)) * (TC_N2 * 16);
          const uint64_t a_h = sdesc(sbase + OFF_A2H + ka, TC_M * 16, 128);
          const uint64_t a_l = sdesc(sbase + OFF_A2L + ka, TC_M * 16, 128);
          const uint64_t b_h = sdesc(sbase + OFF_B2H + kb, TC_N2 * 16, 128);
          const uint64_t b_l = sdesc(sbase + OFF_B2L + kb, TC_N2 * 16, 128);
          mma_tf32(tmem + TC_D2_COL, a_h, b_h, ID2, (pass > 0 || s > 0));
          mma_tf32(tmem + TC_D2_COL, a_h, b_l, ID2, 1);
          mma_tf32(tmem + TC_D2_COL, a_l, b_h, ID2, 1);
        }
        mma_commit(bar2);
      }
      issued2++;
    }
    if (!ok) break;
    if (__syncthreads_or(!bar_wait(bar2, ph2 & 1))) {
      ok = false;
      break;
    }
    ph2++;
    issued2--;
    tc_fence_after();
    // ---- element result: 24 values of tile row tid, added into y
    {
      float yv[24];
      float r[8];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        tmem_ld8(tmem + lane_base + TC_D2_COL + 8 * q, r);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; i++) yv[8 * q + i] = r[i];
      }
      if (valid) {
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
          for (int c = 0; c < 3; c++) atomicAdd(A.y + 3 * node[a] + c, yv[3 * a + c]);
      }
    }
    tc_fence_before();
    __syncthreads();  // D1, D2, A1 and A2 are free for the next tile
  }
  if (!ok) {
    if (tid == 0) {
      atomicOr(A.err, 1u);
      // the MMAs this block issued: wait (bounded) for their commits before freeing
      if (issued1 > 0) bar_wait(bar1, ph1 & 1);
      for (int k = 0; k < issued2; k++) {
        bar_wait(bar2, ph2 & 1);
        ph2++;
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                 : "memory");
}

// Dirichlet rows (MatZeroRowsStencil, VFCartFE.c:1293: rows only): y = x.
__global__ void tc_bc_rows_kernel(const float* __restrict__ x, float* __restrict__ y,
                                  const uint8_t* __restrict__ bc, int64_t N) {
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    const unsigned b = bc[n];
    if (!b) continue;
#pragma unroll
    for (int c = 0; c < 3; c++)
      if ((b >> c) & 1u) y[3 * n + c] = x[3 * n + c];
  }
}

// ---- host: the two constant matrices -------------------------------------------------
// B1 [K1 = 32][N1 = 224] and B2 [K2 = 192][N2 = 32], row-major, from the reference's
// 3-point rule on an hx x hy x hz cell (VFCartFE.c:90-116, 216-269): points
// (1 -+ sqrt(3/5))/2 and 1/2 per axis with weights 5/18, 8/18, 5/18, g = gx + 3 gy + 9 gz,
// local node a = i + 2 j + 4 k, dof 3 a + c.
void tc_tables(double hx, double hy, double hz, double* B1, double* B2) {
  const double pt[3] = {0.5 - VF_TAU, 0.5, 0.5 + VF_TAU}, wt[3] = {VF_W0, VF_W1, VF_W0};
  const double h[3] = {hx, hy, hz}, vol = hx * hy * hz;
  std::memset(B1, 0, sizeof(double) * TC_K1 * TC_N1);
  std::memset(B2, 0, sizeof(double) * TC_K2 * TC_N2);
  for (int g = 0; g < 27; g++) {
    const int gi[3] = {g % 3, (g / 3) % 3, g / 9};
    const double w = wt[gi[0]] * wt[gi[1]] * wt[gi[2]] * vol;
    const int p = g / 9, i = g % 9;
    for (int a = 0; a < 8; a++) {
      const int ai[3] = {a & 1, (a >> 1) & 1, a >> 2};
      double ph[3], dph[3];
      for (int d = 0; d < 3; d++) {
        const double xi = pt[gi[d]];
        ph[d] = ai[d] ? xi : 1.0 - xi;
        dph[d] = (ai[d] ? 1.0 : -1.0) / h[d];
      }
      const double phi = ph[0] * ph[1] * ph[2];
      const double dphi[3] = {dph[0] * ph[1] * ph[2], ph[0] * dph[1] * ph[2], ph[0] * ph[1] * dph[2]};
      auto b1 = [&](int k, int q) -> double& { return B1[k * TC_N1 + 8 * g + q]; };
      auto b2 = [&](int q, int n) -> double& { return B2[(TC_KP * p + 7 * i + q) * TC_N2 + n]; };
      for (int c = 0; c < 3; c++) {
        b1(3 * a + c, 0) = dphi[c];            // tr(grad u)
        b1(3 * a + c, 1 + c) = 2.0 * dphi[c];  // 2 e_cc
        b2(0, 3 * a + c) = w * dphi[c];        // div of the test function
        b2(1 + c, 3 * a + c) = w * dphi[c];    // its e_cc
      }
      // shears: (4) xy, (5) xz, (6) yz
      const int sc[3][2] = {{0, 1}, {0, 2}, {1, 2}};
      for (int q = 0; q < 3; q++) {
        const int c1 = sc[q][0], c2 = sc[q][1];
        b1(3 * a + c1, 4 + q) = dphi[c2];
        b1(3 * a + c2, 4 + q) = dphi[c1];
        b2(4 + q, 3 * a + c1) = w * dphi[c2];
        b2(4 + q, 3 * a + c2) = w * dphi[c1];
      }
      b1(24 + a, 7) = phi;  // v(g)
    }
  }
}

// Round-to-nearest (ties away) to TF32, as cvt.rna.tf32.f32 does.
uint32_t host_tf32(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return u & 0xffffe000u;
  u += 0x1000u;
  return u & 0xffffe000u;
}

// B1 hi, B1 lo, B2 hi, B2 lo in the canonical device layouts (uint32 words).
std::vector<uint32_t> tc_operands(double hx, double hy, double hz) {
  std::vector<double> B1(TC_K1 * TC_N1), B2(TC_K2 * TC_N2);
  tc_tables(hx, hy, hz, B1.data(), B2.data());
  std::vector<uint32_t> out((2 * SZ_B1 + 2 * SZ_B2) / 4, 0u);
  auto put = [&](uint32_t off_hi, uint32_t off_lo, uint32_t o, double b) {
    const uint32_t h = host_tf32((float)b);
    float hf;
    std::memcpy(&hf, &h, 4);
    const uint32_t l = host_tf32((float)(b - (double)hf));
    out[(off_hi + o) / 4] = h;
    out[(off_lo + o) / 4] = l;
  };
  for (int k = 0; k < TC_K1; k++)
    for (int n = 0; n < TC_N1; n++) put(OFF_B1H, OFF_B1L, canon(TC_N1, n, k), B1[k * TC_N1 + n]);
  for (int k = 0; k < TC_K2; k++)
    for (int n = 0; n < TC_N2; n++) put(OFF_B2H, OFF_B2L, canon(TC_N2, n, k), B2[k * TC_N2 + n]);
  return out;
}

}  // namespace
}  // namespace vfgpu

extern "C" int vfgpu_tc_tables(double hx, double hy, double hz, double* B1, double* B2) {
  if (!B1 || !B2 || !(hx > 0) || !(hy > 0) || !(hz > 0))
    return vfgpu::fail(VFGPU_ERR_INVALID, "vfgpu_tc_tables: bad argument");
  vfgpu::tc_tables(hx, hy, hz, B1, B2);
  return VFGPU_OK;
}

extern "C" int vfgpu_u_apply_tc(vfgpu_ctx* c, const float* x, float* y) {
  using namespace vfgpu;
  if (!c || !x || !y) return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_tc: null argument");
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "vfgpu_u_apply_tc: material not set");
  if (c->unilateral) return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_tc: UNILATERAL_NONE only");
  if (!is_device_ptr(x) || !is_device_ptr(y))
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_tc: x and y must be device pointers");
  cudaSetDevice(c->dev);
  int st = ensure_v32(c);
  if (st) return st;
  cudaError_t e = cudaSuccess;
  if (!c->d_tcB) {
    const std::vector<uint32_t> ops = tc_operands(c->hx, c->hy, c->hz);
    e = cudaMalloc(&c->d_tcB, ops.size() * 4);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_tcerr, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemcpy(c->d_tcB, ops.data(), ops.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(c->d_tcerr, 0, sizeof(unsigned));
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_tc: set-up");
    static std::mutex m;
    std::lock_guard<std::mutex> lk(m);
    e = cudaFuncSetAttribute(tc_u_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_tc: kernel attributes");
  }
  TcArgs A{};
  A.x = x;
  A.v = c->V32;
  A.y = y;
  A.B = static_cast<const uint32_t*>(c->d_tcB);
  A.elayer = c->d_elayer;
  A.cellE = c->d_cellE;
  A.P = c->d_params;
  A.err = c->d_tcerr;
  A.nx = c->nx;
  A.ny = c->ny;
  A.nz = c->nz;
  A.ntx = (c->nx - 1 + 31) / 32;
  A.nty = (c->ny - 1 + TC_TY - 1) / TC_TY;
  A.ntiles = (long long)A.ntx * A.nty * (c->nz - 1);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->dev);
  const int grid = (int)std::min<long long>(A.ntiles, nsm);
  const int64_t n3 = 3 * (int64_t)c->N;
  e = cudaMemsetAsync(y, 0, n3 * sizeof(float), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_tcerr, 0, sizeof(unsigned), c->stream);  // this call's flag
  if (e == cudaSuccess) {
    tc_u_apply_kernel<<<grid, 128, TC_SMEM, c->stream>>>(A);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && c->bcU_bits) {
    tc_bc_rows_kernel<<<592, 256, 0, c->stream>>>(x, y, c->bcU_bits, (int64_t)c->N);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_tc");
  return VFGPU_OK;
}

extern "C" int vfgpu_tc_error(vfgpu_ctx* c, int* flagged) {
  using namespace vfgpu;
  if (!c || !flagged) return fail(VFGPU_ERR_INVALID, "vfgpu_tc_error: null argument");
  unsigned h = 0;
  if (c->d_tcerr) {
    cudaError_t e = cudaMemcpy(&h, c->d_tcerr, sizeof h, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_tc_error");
  }
  *flagged = h ? 1 : 0;
  return VFGPU_OK;
}
