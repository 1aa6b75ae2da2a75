// tile_engine.cuh -- the z-marching tile schedule shared by the matrix-free
// operators (U: 3 dofs per node, V: 1 dof per node).
//
// The grid's elements are cut into xy tiles of 32 (x, one warp) x TY (y, TY warps)
// elements; a (tile, node plane) pair is one unit of work, and the ntx nty nz units,
// taken column by column (all planes of tile 0, then tile 1, ...), are shared evenly
// by one wave of blocks: block b takes units [U b / n, U (b + 1) / n), cut at column
// ends into segments.  A segment marches up its planes: per element layer, node
// planes of the tile's 33 x (TY+1) node box stream through a 4-slot shared-memory
// ring by asynchronous copies (cp.async, two planes ahead), each thread computes its
// element's 8 x NC corner contributions (Op::element), those go to shared memory,
// and node-owner threads sum the (up to 4) xy-contributions in a fixed order; the
// z-direction sum is carried in registers.  A segment recomputes the element layer
// below its first plane, so the result does not depend on the split.  Nodes on the
// seams between xy-tiles get partial sums from 2 or 4 tiles, written to a seam buffer
// and summed in a fixed order by seam_fixup_kernel.  The result is deterministic (no
// atomics).
//
// Op supplies:  NC, NIN (per-node inputs staged in smem), EPT (elements per
//   thread: 1, or 2 for an operator that evaluates two y-adjacent elements at once
//   in the two lanes of packed FP32 instructions), the Args type with
//   x/y/seamX/seamY/nx/ny/nz/ntx/nty members, and
//   node_src(A, n, src[NIN]) (global addresses of a node's inputs),
//   element(A, L, ex, ey, ez, in[8][NIN], out[8][NC]) (EPT = 1) or
//   element_multi(A, L, ex, ey[EPT], ez, ok[EPT], in[EPT][8][NIN], out[EPT][8][NC])
//   (EPT > 1; out[e] must be 0 where ok[e] is false),
//   finish_node<DOT>(A, n, val[NC]) (writes y, applying Dirichlet rows / masks; with
//   DOT returns the node's x.y), node_flags(A, n) and finish_node_in<DOT>(A, n, val,
//   flags, xin[NC]) (the same from flags loaded ahead and the node's inputs from the
//   plane ring), and an
//   optional A.skip flag that turns a launch into a no-op (set by a converged CG,
//   so that a queued batch of iterations costs nothing once it is done), LIST:
//   -1, or the unit list (A.ur, A.ustart, A.utotal) the operator's launches take when
//   the list is given -- the U operator's units split by phase field over two
//   launches, each with its own wave of blocks (unit lists 0 and 1) -- and PLANES_TMA:
//   node planes by cp.async values (false) or, for an operator with the U inputs
//   (interlaced x, v) and tensor maps A.xmap / A.vmap, by 1-D tensor copies per tile
//   row (PlaneBox), completion on one mbarrier per ring slot (bounded waits,
//   A.plane_err).
// An Op with CV > 0 per-cell values (the V operator's 27 Gauss-point coefficients)
//   supplies cell_map(A) (a 3-D tensor map, box 32 x TY x CV over (ex, ey, CV ez + g))
//   and cell_err(A), and element(..., cc, cs) reads its cell's values from shared
//   memory (cc[g cs]): one thread issues the tensor copy of element layer k + 2 into a
//   2-stage buffer while layer k is computed, completion tracked by an mbarrier per
//   stage.  The wait is bounded: a thread whose wait gives up sets *cell_err, the
//   block stops at that layer's barrier (no further copy is issued), thread 0 waits
//   (bounded again) for the copies still in flight into its stages, and the block
//   returns.
#pragma once

#include <algorithm>
#include <atomic>

#include "common.cuh"

namespace vfgpu {

// TY element rows per tile; an Op with EPT = 2 gives every thread two y-adjacent
// elements (TY / EPT thread rows).
template <int TY, int EPT = 1> struct Tile {
  static_assert(TY % EPT == 0, "element rows must split evenly over thread rows");
  static constexpr int BX = 33, BY = TY + 1, TR = TY / EPT, NT = 32 * TR;
  static constexpr int NSLOT = (BX * BY + NT - 1) / NT;
};

// Shared memory: a ring of 4 node planes [4][NIN][BY][BX] (during layer k: planes k,
// k+1 read by the elements, plane k read by the node finish after the layer barrier,
// plane k+2 landing, plane k+3 in flight into the slot plane k-1 left) and SCS buffers
// of element corner contributions summed along x [SCS][4*NC][TY][33] (corner pair
// j + 2 kk of element row w at node column l: the i = 1 corner of element l - 1 plus the
// i = 0 corner of element l, added in registers after a warp shuffle):
// two (layer k + 1's elements are written while layer k's node sums still read) where
// MINB blocks of that size fit an SM, else one, with a second barrier per layer.
constexpr int kRing = 4;
// Tensor-copied node planes (Op::PLANES_TMA: the interlaced x, 3 values per node, and v):
// a ring slot holds BY rows of x, then BY rows of v; each row is one 1-D tensor box that
// starts at the row's first value rounded down to 16 bytes (A values), so XBOX / VBOX
// values cover the row's 33 nodes after that shift, at 128-byte row pitches XP / VP.
template <typename T> struct PlaneBox {
  static constexpr int A = 16 / (int)sizeof(T);
  static constexpr int XBOX = (99 + A - 1 + A - 1) / A * A, VBOX = (33 + A - 1 + A - 1) / A * A;
  static constexpr int XP = (XBOX * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  static constexpr int VP = (VBOX * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
};
template <class Op, int TY> constexpr size_t ring_bytes() {
  using T = typename Op::T;
  if constexpr (Op::PLANES_TMA)
    return sizeof(T) * kRing * Tile<TY>::BY * (PlaneBox<T>::XP + PlaneBox<T>::VP);
  else
    return sizeof(T) * kRing * Op::NIN * Tile<TY>::BX * Tile<TY>::BY;
}
template <class Op, int TY, int SCS = 2> constexpr size_t sc_bytes() {
  return sizeof(typename Op::T) * SCS * 4 * Op::NC * 33 * TY;
}
// ring, corner buffers and (PLANES_TMA) one mbarrier per ring slot
template <class Op, int TY, int SCS = 2> constexpr size_t tile_base_bytes() {
  return ring_bytes<Op, TY>() + sc_bytes<Op, TY, SCS>() + (Op::PLANES_TMA ? 8 * kRing : 0);
}
template <class Op, int TY, int MINB> constexpr int sc_stages() {
  return (Op::CV > 0 || MINB * (tile_base_bytes<Op, TY, 2>() + 1024) <= 228 * 1024) ? 2 : 1;
}
// Per-cell value stages (Op::CV > 0): [kCellStages][CV][TY][32] at a 128-byte aligned
// offset, then one 8-byte mbarrier per stage.
constexpr int kCellStages = 2;
template <class Op, int TY> constexpr size_t cell_off() { return (tile_base_bytes<Op, TY>() + 127) & ~size_t(127); }
template <class Op, int TY> constexpr size_t cell_stage_bytes() {
  return sizeof(typename Op::T) * Op::CV * TY * 32;
}
template <class Op, int TY, int MINB> constexpr size_t tile_smem_bytes() {
  if constexpr (Op::CV > 0)
    return cell_off<Op, TY>() + kCellStages * cell_stage_bytes<Op, TY>() + kCellStages * 8;
  else
    return tile_base_bytes<Op, TY, sc_stages<Op, TY, MINB>()>();
}

// mbarrier and tensor-copy primitives (one thread issues; every thread may wait).
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"((unsigned)__cvta_generic_to_shared(bar)),
               "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"((unsigned)__cvta_generic_to_shared(bar)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(bar)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"((unsigned)__cvta_generic_to_shared(bar))
               : "memory");
}
// Waits for the phase with the given parity to complete; gives up after `limit` cycles
// (by default ~2e9, about a second), flags *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned* err,
                                          long long limit = 2000000000ll) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) {
      if (err) atomicOr(err, 1u);
      return false;
    }
  }
}
// 3-D tiled tensor copy global -> shared (no multicast), completion on bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"((unsigned)__cvta_generic_to_shared(bar))
      : "memory");
}

// 1-D tiled tensor copy global -> shared (no multicast), completion on bar; x: the first
// element of the box (its byte offset a multiple of 16).
__device__ __forceinline__ void tma_load_1d(void* dst, const CUtensorMap* map, int x, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2}], [%3];\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
      "l"(map), "r"(x), "r"((unsigned)__cvta_generic_to_shared(bar))
      : "memory");
}

// Asynchronous global -> shared copy of one 4- or 8-byte value (LDGSTS); with
// valid == false nothing is read and the destination is zero-filled.
template <typename T>
__device__ __forceinline__ void cp_async_val(T* smem, const T* gmem, bool valid) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte values");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(valid ? 8 : 0) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// DOT: also write this block's share of x.y to A.dot (the CG's p.w); a separate
// instantiation, so that plain applies carry none of its registers.
template <class Op, int TY, int MINB, bool DOT>
__global__ void __launch_bounds__(32 * TY / Op::EPT, MINB)
    tile_apply_kernel(const __grid_constant__ typename Op::Args A, const LayerTable L) {
  using T = typename Op::T;
  using G = Tile<TY, Op::EPT>;
  constexpr int EPT = Op::EPT;
  constexpr int NC = Op::NC, NIN = Op::NIN;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int SCS = sc_stages<Op, TY, MINB>();
  T* sx = reinterpret_cast<T*>(smem_raw);  // [kRing][NIN][BY][BX], or the PlaneBox rows
  T* sc = reinterpret_cast<T*>(smem_raw + ring_bytes<Op, TY>());  // [SCS][4*NC][TY][33]
  [[maybe_unused]] uint64_t* pbar = nullptr;  // PLANES_TMA: one mbarrier per ring slot
  if constexpr (Op::PLANES_TMA)
    pbar = reinterpret_cast<uint64_t*>(smem_raw + ring_bytes<Op, TY>() + sc_bytes<Op, TY, SCS>());
  const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
  const int nx = A.nx, ny = A.ny, nz = A.nz, nex = nx - 1, ney = ny - 1;
  // This block's share of the work: node planes [U b / n, U (b + 1) / n) of the
  // U = ntx nty nz (xy tile, node plane) units taken column by column, cut at column
  // ends into segments (a segment recomputes the element layer below its first plane,
  // so the result does not depend on the split) -- or, with unit list Op::LIST, of the
  // U units of the list's runs, cut at run ends.
  [[maybe_unused]] const int4* runs = nullptr;
  [[maybe_unused]] int run = 0;
  int64_t U = (int64_t)A.ntx * A.nty * nz;
  if constexpr (Op::LIST >= 0) {
    runs = A.ur[Op::LIST];
    if (runs) U = A.utotal[Op::LIST];
  }
  const int64_t u_begin = U * blockIdx.x / gridDim.x, u_end = U * (blockIdx.x + 1) / gridDim.x;
  if (u_begin >= u_end) {
    if (DOT && threadIdx.x + threadIdx.y == 0) A.dot[blockIdx.x] = 0.;
    return;
  }
  if (A.skip && *A.skip) return;  // converged solve: uniform early exit, before any barrier
  double dacc = 0.;  // this thread's share of x.y over the nodes it finishes (A.dot)
  [[maybe_unused]] T* cbuf = nullptr;
  [[maybe_unused]] uint64_t* cbar = nullptr;
  if constexpr (Op::CV > 0) {
    cbuf = reinterpret_cast<T*>(smem_raw + cell_off<Op, TY>());
    cbar = reinterpret_cast<uint64_t*>(smem_raw + cell_off<Op, TY>() + kCellStages * cell_stage_bytes<Op, TY>());
  }

  // Returns false if a bounded wait on the per-cell copies gave up (the block then
  // stops: see the layer barrier).
  auto run_segment = [&](const int bx, const int by, const int z0, const int z1) -> bool {
  const int X0 = bx * 32, Y0 = by * TY;
  const int kf = max(z0 - 1, 0), kl = min(z1, nz - 1) - 1;

#define SXA(buf, comp, w, l) sx[(((buf) * NIN + (comp)) * G::BY + (w)) * G::BX + (l)]
#define SCA(b, q, w, l) sc[(((b) * 4 * NC + (q)) * TY + (w)) * 33 + (l)]

  // The x-sums of element row w's corner contributions yc[a], a = i + 2 j + 4 kk, into
  // corner-pair rows q = j + 2 kk: node column lane gets (element lane - 1, i = 1) +
  // (element lane, i = 0), column 32 the i = 1 corners of element 31 (whole warp).
  auto store_xsums = [&](int sbuf, int w, const T (&yc)[8][NC]) {
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const T own = yc[2 * q][c], rt = yc[2 * q + 1][c];
        const T left = __shfl_up_sync(0xffffffffu, rt, 1);
        SCA(sbuf, q * NC + c, w, lane) = lane > 0 ? left + own : own;
        if (lane == 31) SCA(sbuf, q * NC + c, w, 32) = rt;
      }
  };

  // input q of the node in tile row w, column l of plane kz, from ring slot buf (with
  // PLANES_TMA: x component q < 3 or v, at the row's 16-byte shift, which only the low
  // bits of the row's first node index decide)
  auto rv = [&](int buf, int kz, int q, int w, int l) -> T {
    if constexpr (Op::PLANES_TMA) {
      using PB = PlaneBox<T>;
      const unsigned n0 = ((unsigned)kz * (unsigned)ny + (unsigned)(Y0 + w)) * (unsigned)nx + (unsigned)X0;
      if (q < 3) return sx[(buf * G::BY + w) * PB::XP + 3 * l + q + (int)((3u * n0) & (PB::A - 1))];
      return sx[kRing * G::BY * PB::XP + (buf * G::BY + w) * PB::VP + l + (int)(n0 & (PB::A - 1))];
    } else {
      return SXA(buf, q, w, l);
    }
  };

  // issue the copies of node plane kz into ring slot buf: one cp.async group, or
  // (PLANES_TMA) two tensor copies per tile row from warp 0, completing on pbar[buf]
  auto fetch_plane = [&](int buf, int kz) {
    if constexpr (Op::PLANES_TMA) {
      using PB = PlaneBox<T>;
      if (wy == 0) {
        const int rows = min(G::BY, ny - Y0);
        if (lane == 0)
          mbar_expect_tx(&pbar[buf], (unsigned)(rows * (PB::XBOX + PB::VBOX) * sizeof(T)));
        __syncwarp();
        if (lane < rows) {
          const int64_t n0 = ((int64_t)kz * ny + Y0 + lane) * nx + X0, e0 = 3 * n0;
          tma_load_1d(sx + (buf * G::BY + lane) * PB::XP, &A.xmap, (int)(e0 - (e0 & (PB::A - 1))),
                      &pbar[buf]);
          tma_load_1d(sx + kRing * G::BY * PB::XP + (buf * G::BY + lane) * PB::VP, &A.vmap,
                      (int)(n0 - (n0 & (PB::A - 1))), &pbar[buf]);
        }
      }
    } else {
      for (int s = tid; s < G::BX * G::BY; s += G::NT) {
        const int l = s % G::BX, w = s / G::BX, X = X0 + l, Y = Y0 + w;
        const bool in = X < nx && Y < ny;
        const T* src[NIN];
        Op::node_src(A, in ? node_index(X, Y, kz, nx, ny) : 0, src);
#pragma unroll
        for (int q = 0; q < NIN; q++) cp_async_val(&SXA(buf, q, w, l), src[q], in);
      }
      cp_async_commit();
    }
  };
  // PLANES_TMA: the slot and phase parity of plane kz's copy in this segment
  [[maybe_unused]] auto pslot = [&](int kz) { return (kz - kf) % kRing; };
  [[maybe_unused]] auto pphase = [&](int kz) { return (unsigned)(((kz - kf) / kRing) & 1); };

  // fl: the node's flags (loaded ahead), buf: the ring slot holding plane z
  auto emit = [&](int l, int w, int X, int Y, int z, const T (&val)[NC], unsigned fl, int buf) {
    const bool left = (l == 0 && bx > 0), right = (l == 32 && bx < A.ntx - 1);
    const bool bot = (w == 0 && by > 0), top = (w == TY && by < A.nty - 1);
    if (!(left || right || bot || top)) {
      T xin[NC];
#pragma unroll
      for (int c = 0; c < NC; c++) xin[c] = rv(buf, z, c, w, l);
      dacc += Op::template finish_node_in<DOT>(A, node_index(X, Y, z, nx, ny), val, fl, xin);
    } else if (left || right) {
      const int i = left ? bx : bx + 1;
      const int slot = (bot ? 2 : 0) + (left ? 1 : 0);
      T* p = A.seamX + ((((int64_t)(i - 1) * nz + z) * ny + Y) * 4 + slot) * NC;
#pragma unroll
      for (int c = 0; c < NC; c++) p[c] = val[c];
    } else {
      const int j = bot ? by : by + 1;
      T* p = A.seamY + ((((int64_t)(j - 1) * nz + z) * nx + X) * 2 + (bot ? 1 : 0)) * NC;
#pragma unroll
      for (int c = 0; c < NC; c++) p[c] = val[c];
    }
  };

  T carry[G::NSLOT][NC];
#pragma unroll
  for (int si = 0; si < G::NSLOT; si++)
#pragma unroll
    for (int c = 0; c < NC; c++) carry[si][c] = T(0);

  // Pipeline: planes kf, kf+1 resident before the first layer; during layer k the
  // copy of plane k+2 is in flight; one barrier per layer publishes plane k+2 and
  // the corner contributions of layer k together.
  [[maybe_unused]] bool gave_up = false;
  if constexpr (Op::PLANES_TMA) {
    if (tid == 0) {
      for (int st = 0; st < kRing; st++) mbar_init(&pbar[st], 1);
      mbar_fence_init();
    }
    __syncthreads();  // initialised before any copy or wait
  }
  fetch_plane(0, kf);
  fetch_plane(1, kf + 1);
  // per-cell values of layers kf, kf + 1 (CV > 0): issued before the first barrier,
  // which also publishes the mbarrier initialisation
  [[maybe_unused]] auto fetch_cells = [&](int st, int kz) {
    if constexpr (Op::CV > 0) {
      mbar_expect_tx(&cbar[st], (unsigned)cell_stage_bytes<Op, TY>());
      tma_load_3d(cbuf + (size_t)st * Op::CV * TY * 32, Op::cell_map(A), X0, Y0, Op::CV * kz, &cbar[st]);
    }
  };
  if constexpr (Op::CV > 0) {
    if (tid == 0) {
      for (int st = 0; st < kCellStages; st++) mbar_init(&cbar[st], 1);
      mbar_fence_init();
      for (int st = 0; st < kCellStages; st++)
        if (kf + st <= kl) fetch_cells(st, kf + st);
    }
  }
  if constexpr (Op::PLANES_TMA) {
    // bounded waits; if one gives up the block stops (thread 0 first waits, bounded again,
    // for the copies in flight into slots 0 and 1) and the launch's results are void
    gave_up = !mbar_wait(&pbar[0], 0u, A.plane_err);
    gave_up = !mbar_wait(&pbar[1], 0u, A.plane_err) || gave_up;
    if (__syncthreads_or(gave_up)) {
      if (tid == 0) {
        mbar_wait(&pbar[0], 0u, nullptr);
        mbar_wait(&pbar[1], 0u, nullptr);
      }
      return false;
    }
  } else {
    cp_async_wait_all();
    __syncthreads();
  }
  if (kf + 2 <= kl + 1) fetch_plane(2, kf + 2);
  for (int k = kf; k <= kl; k++) {
    const int r0 = (k - kf) % kRing, r1 = (k - kf + 1) % kRing, sb = SCS == 2 ? (k - kf) & 1 : 0;
    // the flags of the nodes this thread finishes after the layer (plane k), loaded now
    // so that the finish does not wait for them
    unsigned nfl[G::NSLOT];
#pragma unroll
    for (int si = 0; si < G::NSLOT; si++) {
      const int s = tid + si * G::NT, l = s % G::BX, w = s / G::BX, X = X0 + l, Y = Y0 + w;
      nfl[si] = (k >= z0 && s < G::BX * G::BY && X < nx && Y < ny)
                    ? Op::node_flags(A, node_index(X, Y, k, nx, ny)) : 0u;
    }
    const int ex = X0 + lane;
    if constexpr (EPT == 1) {
      const int ey = Y0 + wy;
      T yc[8][NC];
      if constexpr (Op::CV > 0)
        gave_up = !mbar_wait(&cbar[(k - kf) % kCellStages], ((k - kf) / kCellStages) & 1, Op::cell_err(A));
      if (ex < nex && ey < ney) {
        T in[8][NIN];
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
#pragma unroll
          for (int j = 0; j < 2; j++)
#pragma unroll
            for (int i = 0; i < 2; i++) {
              const int a = i + 2 * j + 4 * kk, buf = kk ? r1 : r0;
#pragma unroll
              for (int q = 0; q < NIN; q++) in[a][q] = rv(buf, k + kk, q, wy + j, lane + i);
            }
        if constexpr (Op::CV > 0)
          Op::element(A, L, ex, ey, k, in, yc,
                      cbuf + (size_t)((k - kf) % kCellStages) * Op::CV * TY * 32 + wy * 32 + lane,
                      TY * 32);
        else
          Op::element(A, L, ex, ey, k, in, yc);
      } else {
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
          for (int c = 0; c < NC; c++) yc[a][c] = T(0);
      }
      store_xsums(sb, wy, yc);
    } else {
      // element rows EPT*wy + e, e < EPT (node rows EPT*wy .. EPT*wy + EPT)
      int ey[EPT];
      bool ok[EPT], any = false;
#pragma unroll
      for (int e = 0; e < EPT; e++) {
        ey[e] = Y0 + EPT * wy + e;
        ok[e] = ex < nex && ey[e] < ney;
        any = any || ok[e];
      }
      T yc[EPT][8][NC];
      if (any) {
        T in[EPT][8][NIN];
#pragma unroll
        for (int e = 0; e < EPT; e++)
#pragma unroll
          for (int kk = 0; kk < 2; kk++)
#pragma unroll
            for (int j = 0; j < 2; j++)
#pragma unroll
              for (int i = 0; i < 2; i++) {
                const int a = i + 2 * j + 4 * kk, buf = kk ? r1 : r0;
#pragma unroll
                for (int q = 0; q < NIN; q++) in[e][a][q] = rv(buf, k + kk, q, EPT * wy + e + j, lane + i);
              }
        Op::element_multi(A, L, ex, ey, k, ok, in, yc);
      } else {
#pragma unroll
        for (int e = 0; e < EPT; e++)
#pragma unroll
          for (int a = 0; a < 8; a++)
#pragma unroll
            for (int c = 0; c < NC; c++) yc[e][a][c] = T(0);
      }
#pragma unroll
      for (int e = 0; e < EPT; e++) store_xsums(sb, EPT * wy + e, yc[e]);
    }
    if constexpr (Op::PLANES_TMA) {  // plane k+2 has landed (bounded)
      if (k + 2 <= kl + 1 && !mbar_wait(&pbar[pslot(k + 2)], pphase(k + 2), A.plane_err)) gave_up = true;
    } else {
      cp_async_wait_all();  // this thread's copies of plane k+2 have landed
    }
    if constexpr (Op::CV > 0) {
      // ... and everyone's; corner contributions of layer k visible.  If any thread's
      // wait on layer k's values gave up, the whole block stops here: no further copy
      // is issued, thread 0 waits (bounded) for the tensor copies still in flight into
      // the stages of layers k and k + 1, and the launch's results are void (the host
      // sees *cell_err).
      if (__syncthreads_or(gave_up)) {
        if (tid == 0) {
          mbar_wait(&cbar[(k - kf) % kCellStages], ((k - kf) / kCellStages) & 1, nullptr);
          if (k + 1 <= kl)
            mbar_wait(&cbar[(k + 1 - kf) % kCellStages], ((k + 1 - kf) / kCellStages) & 1, nullptr);
        }
        return false;
      }
    } else if constexpr (Op::PLANES_TMA) {
      // ... corner contributions of layer k visible; if a wait on plane k+2 gave up the
      // block stops, thread 0 waiting (bounded) for that plane's copies in flight
      if (__syncthreads_or(gave_up)) {
        if (tid == 0 && k + 2 <= kl + 1) mbar_wait(&pbar[pslot(k + 2)], pphase(k + 2), nullptr);
        return false;
      }
    } else {
      __syncthreads();    // ... and everyone's; corner contributions of layer k visible
    }
    if (k + 3 <= kl + 1) fetch_plane((k + 3 - kf) % kRing, k + 3);  // the slot of plane k - 1
    if constexpr (Op::CV > 0)  // layer k's stage is no longer read
      if (tid == 0 && k + kCellStages <= kl) fetch_cells((k - kf) % kCellStages, k + kCellStages);
#pragma unroll
    for (int si = 0; si < G::NSLOT; si++) {
      const int s = tid + si * G::NT;
      if (s >= G::BX * G::BY) continue;
      const int l = s % G::BX, w = s / G::BX, X = X0 + l, Y = Y0 + w;
      if (X >= nx || Y >= ny) continue;
      T p0[NC], p1[NC];
#pragma unroll
      for (int c = 0; c < NC; c++) p0[c] = p1[c] = T(0);
#pragma unroll
      for (int dw = 0; dw < 2; dw++) {
        const int ew = w - 1 + dw, j = 1 - dw;
        if (ew < 0 || ew >= TY) continue;
#pragma unroll
        for (int c = 0; c < NC; c++) {
          p0[c] += SCA(sb, j * NC + c, ew, l);
          p1[c] += SCA(sb, (j + 2) * NC + c, ew, l);
        }
      }
      if (k >= z0) {
        T val[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) val[c] = carry[si][c] + p0[c];
        emit(l, w, X, Y, k, val, nfl[si], r0);
      }
#pragma unroll
      for (int c = 0; c < NC; c++) carry[si][c] = p1[c];
    }
    if constexpr (SCS == 1) __syncthreads();  // the next layer rewrites the one buffer
  }
  if (z1 == nz) {
#pragma unroll
    for (int si = 0; si < G::NSLOT; si++) {
      const int s = tid + si * G::NT;
      if (s >= G::BX * G::BY) continue;
      const int l = s % G::BX, w = s / G::BX, X = X0 + l, Y = Y0 + w;
      if (X >= nx || Y >= ny) continue;
      emit(l, w, X, Y, nz - 1, carry[si], Op::node_flags(A, node_index(X, Y, nz - 1, nx, ny)),
           (nz - 1 - kf) % kRing);
    }
  }
  return true;
  };  // run_segment

  if constexpr (Op::LIST >= 0)
    if (runs) run = A.ustart[Op::LIST][blockIdx.x];
  for (int64_t u = u_begin; u < u_end;) {
    int col, z0, z1;
    if (runs) {
      const int4 R = runs[run++];  // the run holding unit u
      col = R.x;
      z0 = R.y + (int)(u - R.w);
      z1 = (int)std::min<int64_t>(R.z, R.y + (u_end - R.w));
    } else {
      col = (int)(u / nz);
      z0 = (int)(u % nz);
      const int64_t left = u_end - u;
      z1 = left < (int64_t)(nz - z0) ? z0 + (int)left : nz;
    }
    if (!run_segment(col % A.ntx, col / A.ntx, z0, z1)) break;  // block-uniform
    u += z1 - z0;
    if (u < u_end) {
      __syncthreads();  // the next segment reuses the shared-memory buffers
      if constexpr (Op::CV > 0)  // every phase of the stages completed: re-armed by the next init
        if (tid == 0)
          for (int st = 0; st < kCellStages; st++) mbar_inval(&cbar[st]);
      if constexpr (Op::PLANES_TMA)  // every plane copied was waited for
        if (tid == 0)
          for (int st = 0; st < kRing; st++) mbar_inval(&pbar[st]);
    }
  }
  if constexpr (DOT) {
    __syncthreads();  // the shared-memory buffers are no longer read
    const double bs = block_sum_dbl(dacc, reinterpret_cast<double*>(smem_raw));
    if (tid == 0) A.dot[blockIdx.x] = bs;
  }
#undef SXA
#undef SCA
}

// Sums the 2 (or 4 where an x-seam crosses a y-seam) tile partials of every
// seam node in a fixed order and finishes the node (Op::finish_node); with A.dot,
// block b's share of x.y goes to A.dot[dot_base + b].
template <class Op, bool DOT>
__global__ void __launch_bounds__(256) seam_fixup_kernel(const typename Op::Args A, int TY, int dot_base) {
  using T = typename Op::T;
  constexpr int NC = Op::NC;
  __shared__ double red[32];
  const int nx = A.nx, ny = A.ny, nz = A.nz;
  if (A.skip && *A.skip) return;
  double dacc = 0.;
  const int64_t nxs = (int64_t)(A.ntx - 1) * nz * ny;
  const int64_t nys = (int64_t)(A.nty - 1) * nz * nx;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nxs + nys;
       t += (int64_t)gridDim.x * blockDim.x) {
    T val[NC];
    int64_t n;
    if (t < nxs) {
      const int Y = (int)(t % ny);
      const int64_t r = t / ny;
      const int z = (int)(r % nz), i = (int)(r / nz) + 1;
      const bool onY = (Y % TY == 0) && (Y > 0) && (Y / TY < A.nty);
      const T* p = A.seamX + t * 4 * NC;
#pragma unroll
      for (int c = 0; c < NC; c++)
        val[c] = onY ? ((p[c] + p[NC + c]) + p[2 * NC + c]) + p[3 * NC + c] : p[c] + p[NC + c];
      n = node_index(32 * i, Y, z, nx, ny);
    } else {
      const int64_t u = t - nxs;
      const int X = (int)(u % nx);
      const int64_t r = u / nx;
      const int z = (int)(r % nz), j = (int)(r / nz) + 1;
      if (X % 32 == 0 && X > 0 && X / 32 < A.ntx) continue;
      const T* p = A.seamY + u * 2 * NC;
#pragma unroll
      for (int c = 0; c < NC; c++) val[c] = p[c] + p[NC + c];
      n = node_index(X, TY * j, z, nx, ny);
    }
    dacc += Op::template finish_node<DOT>(A, n, val);
  }
  if constexpr (DOT) {
    const double bs = block_sum_dbl(dacc, red);
    if (threadIdx.x == 0) A.dot[dot_base + blockIdx.x] = bs;
  }
}


// Launch plan: xy tiles of 32 x ty elements, the blocks of one launch (one wave of
// ctas_per_sm blocks per SM, or one unit per block on small grids) and the seam buffer
// sizes in elements of T.
struct TilePlan {
  int ty, ntx, nty;
  int ncta;
  int ncta0;  // the wave of a split launch's unit list 0 (UOpConst), which may take more
              // blocks per SM; = ncta otherwise
  size_t seamX, seamY;
};

inline TilePlan tile_plan(int nx, int ny, int nz, int ty, int nc, int ctas_per_sm, int num_sms) {
  TilePlan p;
  p.ty = ty;
  p.ntx = (nx - 1 + 31) / 32;
  p.nty = (ny - 1 + ty - 1) / ty;
  const int slots = num_sms * ctas_per_sm, tiles = p.ntx * p.nty;
  const int64_t units = (int64_t)tiles * nz;
  p.ncta = (int)std::max<int64_t>(1, std::min<int64_t>(slots, units));
  p.ncta0 = p.ncta;
  p.seamX = (size_t)(p.ntx - 1) * nz * ny * 4 * nc;
  p.seamY = (size_t)(p.nty - 1) * nz * nx * 2 * nc;
  return p;
}

// Launch shape of the seam fix-up (0 blocks: no seams) and the number of x.y block
// partials one operator launch writes when it accumulates the CG dot.
inline int seam_blocks(const TilePlan& p, int nx, int ny, int nz) {
  const int64_t nseam = (int64_t)(p.ntx - 1) * nz * ny + (int64_t)(p.nty - 1) * nz * nx;
  if (nseam <= 0) return 0;
  return (int)std::min<int64_t>((nseam + 255) / 256, 148 * 8);
}
inline int tile_dot_count(const TilePlan& p, int nx, int ny, int nz) {
  return p.ncta + seam_blocks(p, nx, ny, nz);
}

// Opt-in to the dynamic shared memory the kernel needs; done once per device (and
// up front, from vfgpu_create, so that no attribute call happens inside a capture).
// The per-device bits are atomic, so concurrent callers at worst repeat the
// (idempotent) attribute call.
template <class Op, int TY, int MINB> inline std::atomic<unsigned long long> g_tile_attr_set{0};
template <class Op, int TY, int MINB> cudaError_t set_tile_attributes() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (g_tile_attr_set<Op, TY, MINB>.load(std::memory_order_acquire) & bit) return cudaSuccess;
  const int smem = (int)tile_smem_bytes<Op, TY, MINB>();
  e = cudaFuncSetAttribute(tile_apply_kernel<Op, TY, MINB, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(tile_apply_kernel<Op, TY, MINB, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) g_tile_attr_set<Op, TY, MINB>.fetch_or(bit, std::memory_order_release);
  return e;
}

template <class Op, int TY, int MINB>
cudaError_t launch_tile_apply(typename Op::Args A, const TilePlan& p, const LayerTable& L,
                              cudaStream_t s) {
  A.ntx = p.ntx;
  A.nty = p.nty;
  constexpr size_t smem = tile_smem_bytes<Op, TY, MINB>();
  cudaError_t ea = set_tile_attributes<Op, TY, MINB>();
  if (ea != cudaSuccess) return ea;
  dim3 grid(p.ncta), block(32, TY / Op::EPT);
  const int sblocks = seam_blocks(p, A.nx, A.ny, A.nz), base = p.ncta;
  if (A.dot) {
    tile_apply_kernel<Op, TY, MINB, true><<<grid, block, smem, s>>>(A, L);
    if (sblocks > 0) seam_fixup_kernel<Op, true><<<sblocks, 256, 0, s>>>(A, TY, base);
  } else {
    tile_apply_kernel<Op, TY, MINB, false><<<grid, block, smem, s>>>(A, L);
    if (sblocks > 0) seam_fixup_kernel<Op, false><<<sblocks, 256, 0, s>>>(A, TY, base);
  }
  return cudaGetLastError();
}


// An operator split over unit lists 0 (OpF, MINBF blocks per SM, a wave of p.ncta0) and 1
// (OpG, MINB, a wave of p.ncta; it also finishes the seams): the two waves in turn, then
// the seam fix-up.  With A.dot the x.y block partials go to A.dot[0, ncta0) (OpF),
// [ncta0, ncta0 + ncta) (OpG) and from ncta0 + ncta on (seams): tile_dot_count + ncta0
// of them.
template <class OpF, class OpG, int TY, int MINBF, int MINB>
cudaError_t launch_tile_apply_split(typename OpG::Args A, const TilePlan& p, const LayerTable& L,
                                    cudaStream_t s) {
  static_assert(OpF::LIST == 0 && OpG::LIST == 1 && OpG::EPT == 1, "unit lists 0, 1");
  A.ntx = p.ntx;
  A.nty = p.nty;
  constexpr size_t smemF = tile_smem_bytes<OpF, TY, MINBF>(), smemG = tile_smem_bytes<OpG, TY, MINB>();
  cudaError_t ea = set_tile_attributes<OpF, TY, MINBF>();
  if (ea == cudaSuccess) ea = set_tile_attributes<OpG, TY, MINB>();
  if (ea != cudaSuccess) return ea;
  const dim3 blockF(32, TY / OpF::EPT), block(32, TY);
  const int sblocks = seam_blocks(p, A.nx, A.ny, A.nz), base = p.ncta0 + p.ncta;
  typename OpG::Args AG = A;
  if (AG.dot) AG.dot += p.ncta0;
  if (A.dot) {
    tile_apply_kernel<OpF, TY, MINBF, true><<<p.ncta0, blockF, smemF, s>>>(A, L);
    tile_apply_kernel<OpG, TY, MINB, true><<<p.ncta, block, smemG, s>>>(AG, L);
    if (sblocks > 0) seam_fixup_kernel<OpG, true><<<sblocks, 256, 0, s>>>(A, TY, base);
  } else {
    tile_apply_kernel<OpF, TY, MINBF, false><<<p.ncta0, blockF, smemF, s>>>(A, L);
    tile_apply_kernel<OpG, TY, MINB, false><<<p.ncta, block, smemG, s>>>(AG, L);
    if (sblocks > 0) seam_fixup_kernel<OpG, false><<<sblocks, 256, 0, s>>>(A, TY, base);
  }
  return cudaGetLastError();
}

}  // namespace vfgpu
