// apply.cu -- instantiations of the tile engine for the U and V operators.
#include <mutex>
#include <type_traits>

#include "kernels.h"
#include "ops.cuh"

namespace vfgpu {

// FP64 U operator tiles: 32 x U64_TY elements (1 CTA per SM: ~250 registers per thread).
// 12 rows (12 warps per SM at 168 registers, with 288 bytes of spills) measured slower
// on B200: 0.280 against 0.253 ms at 129^3, 0.814 against 0.733 ms at 193^3.
#ifndef VFGPU_U64_TY
#define VFGPU_U64_TY 8
#endif
constexpr int U_TY = 8, U64_TY = VFGPU_U64_TY, V_TY = kVTileY;
// Blocks per SM of the FP64 U operator: 1 (~250 registers, two corner-contribution
// buffers) or, as a build option, 2 (128 registers: the row closed form of the
// non-constant elements spills; one buffer and a second barrier per layer).
#ifndef VFGPU_U64_MINB
#define VFGPU_U64_MINB 1
#endif
constexpr int U64_MINB = VFGPU_U64_MINB;
// The fixed-weight U kernel of a split launch (UOpConst: fewer registers, and the x-summed
// corner buffers leave room for both stages) takes more blocks per SM than the general
// one: 2 (FP64) and 3 (FP32) measured 0.117 / 0.089 ms at 129^3 on the penny field against
// 0.134 / 0.091 ms with the general kernel's 1 and 2.
#ifndef VFGPU_U64C_MINB
#define VFGPU_U64C_MINB 2
#endif
#ifndef VFGPU_U32C_MINB
#define VFGPU_U32C_MINB 3
#endif
// The FP32 fixed-weight wave on packed two-lane FP32 (UOpF2Const: two element rows per
// thread, 4 warps per block; the same bits as the scalar UOpConst<float>) or scalar.
// Measured at 129^3 on the penny field, whole FP32 apply: packed at 4 blocks per SM
// (118-126 registers) 0.0855 ms, at 3 0.0905, at 5 (spilling) 0.0879, at 2 0.0981;
// scalar at 3 blocks per SM 0.0900 ms.
#ifndef VFGPU_U32C_PACKED
#define VFGPU_U32C_PACKED 1
#endif
#ifndef VFGPU_U32C2_MINB
#define VFGPU_U32C2_MINB 4
#endif
constexpr bool kU32CPacked = VFGPU_U32C_PACKED != 0;
constexpr int U64C_MINB = VFGPU_U64C_MINB,
              U32C_MINB = kU32CPacked ? VFGPU_U32C2_MINB : VFGPU_U32C_MINB;
using U32COp = std::conditional_t<kU32CPacked, UOpF2Const<false>, UOpConst<float>>;
using U32COpC = std::conditional_t<kU32CPacked, UOpF2Const<true>, UOpConst<float, true>>;
// V tiles carry 2 stages of 27 coefficients per cell in shared memory: 75 KB (FP32,
// 2 CTAs per SM) or 150 KB (FP64, 1 CTA per SM).
constexpr int V64_MINB = 1, V32_MINB = 2;
// FP32 U operator: scalar UOp<float> (2 CTAs of 8 warps per SM) by default.  The
// packed two-lane variant (UOpF2: two elements per thread, half the arithmetic
// instructions) is kept as a build option; it needs 242 registers, so one CTA of
// 8 warps per SM, and measured slower on B200: 0.185 ms against 0.161 ms at 129^3,
// 0.353 ms against 0.298 ms at 161^3 (16 element rows; 0.189 / 0.339 ms with 8).
#ifndef VFGPU_U32_PACKED
#define VFGPU_U32_PACKED 0
#endif
#ifndef VFGPU_U32_PACKED_TY
#define VFGPU_U32_PACKED_TY 16
#endif
constexpr bool kU32Packed = VFGPU_U32_PACKED != 0;
constexpr int U32_TY = kU32Packed ? VFGPU_U32_PACKED_TY : U_TY;
#ifndef VFGPU_U32_MINB
#define VFGPU_U32_MINB 2
#endif
constexpr int U32_MINB = kU32Packed ? (VFGPU_U32_PACKED_TY == 16 ? 1 : 2) : VFGPU_U32_MINB;
using U32Op = std::conditional_t<kU32Packed, UOpF2, UOp<float>>;
using U32OpC = std::conditional_t<kU32Packed, UOpF2, UOp<float, true>>;

// Cubic cells take the U element with every 1/h folded into the row weight.
template <typename T> bool cubic(const UApplyArgs<T>& A) { return A.ihx == A.ihy && A.ihy == A.ihz; }

cudaError_t apply_kernel_attributes() {
  static std::mutex m;  // contexts may be created from several threads
  std::lock_guard<std::mutex> lk(m);
  cudaError_t e = set_tile_attributes<UOp<double>, U64_TY, U64_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<UOp<double, true>, U64_TY, U64_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<UOpConst<double>, U64_TY, U64C_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<UOpConst<double, true>, U64_TY, U64C_MINB>();
  if constexpr (!kU32Packed) {
    if (e == cudaSuccess) e = set_tile_attributes<U32COp, U32_TY, U32C_MINB>();
    if (e == cudaSuccess) e = set_tile_attributes<U32COpC, U32_TY, U32C_MINB>();
  }
  if (e == cudaSuccess) e = set_tile_attributes<U32Op, U32_TY, U32_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<U32OpC, U32_TY, U32_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<UOpNC<double>, U64_TY, 1>();
  if (e == cudaSuccess) e = set_tile_attributes<UOpNC<float>, U_TY, 2>();
  if (e == cudaSuccess) e = set_tile_attributes<VOp<double>, V_TY, V64_MINB>();
  if (e == cudaSuccess) e = set_tile_attributes<VOp<float>, V_TY, V32_MINB>();
  return e;
}

using TensorEncode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);
// cuTensorMapEncodeTiled from the driver (null if it has none)
static TensorEncode tensor_encode() {
  static const TensorEncode fn = []() -> TensorEncode {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<TensorEncode>(f);
  }();
  return fn;
}

cudaError_t vcoef_tensor_map(CUtensorMap* map, const void* coef, int bytes, int nex, int ney, int nez) {
  const TensorEncode encode = tensor_encode();
  if (!encode) return cudaErrorNotSupported;
  const int pitch = vcoef_pitch(nex);
  const cuuint64_t dims[3] = {(cuuint64_t)nex, (cuuint64_t)ney, (cuuint64_t)27 * nez};
  const cuuint64_t strides[2] = {(cuuint64_t)pitch * bytes, (cuuint64_t)pitch * ney * bytes};
  const cuuint32_t box[3] = {32, (cuuint32_t)kVTileY, 27}, estride[3] = {1, 1, 1};
  const CUresult r =
      encode(map, bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
             const_cast<void*>(coef), dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// One CTA waits on an mbarrier whose phase completes (complete = 1: the arrival is
// made) or never does (complete = 0: 16 transaction bytes are expected and no copy is
// issued); the bounded wait sets *err when it gives up.
__global__ void wait_selftest_kernel(unsigned* err, long long limit, int complete) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
    if (complete) mbar_arrive(&bar);
    else mbar_expect_tx(&bar, 16);
  }
  __syncthreads();
  mbar_wait(&bar, 0, err, limit);
}

cudaError_t wait_selftest(long long cycles, int complete, int* timed_out) {
  unsigned* d = nullptr;
  unsigned h = 0;
  cudaError_t e = cudaMalloc(&d, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(unsigned));
  if (e == cudaSuccess) {
    wait_selftest_kernel<<<1, 64>>>(d, cycles, complete);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost);
  cudaFree(d);
  *timed_out = h ? 1 : 0;
  return e;
}

// ------------------------------------------------------------------ unit lists
// cls[(by ntx + bx) (nz - 1) + k] = 1 when every element of tile (bx, by) (32 x TY
// elements) in element layer k has 8 equal nodal v (elements beyond the grid count as
// equal).  One block per tile and run of kClsLayers layers: each thread loads its
// element column's 2 x 2 node quads of the run's kClsLayers + 1 planes at once, then
// votes per layer.
constexpr int kClsLayers = 8;
template <int TY>
__global__ void __launch_bounds__(32 * TY) u_classify_kernel(const double* __restrict__ v,
                                                              uint8_t* __restrict__ cls, int nx,
                                                              int ny, int nez) {
  __shared__ int all[kClsLayers];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  if (tid < kClsLayers) all[tid] = 1;
  const int ex = blockIdx.x * 32 + threadIdx.x, ey = blockIdx.y * TY + threadIdx.y;
  const int k0 = blockIdx.z * kClsLayers;
  const bool in = ex < nx - 1 && ey < ny - 1;
  const int64_t pl = (int64_t)nx * ny;
  const double* w = v + (in ? (int64_t)k0 * pl + (int64_t)ey * nx + ex : 0);
  double q[kClsLayers + 1][4];
#pragma unroll
  for (int i = 0; i <= kClsLayers; i++) {
    const bool ld = in && k0 + i <= nez;
    q[i][0] = ld ? w[i * pl] : 0.;
    q[i][1] = ld ? w[i * pl + 1] : 0.;
    q[i][2] = ld ? w[i * pl + nx] : 0.;
    q[i][3] = ld ? w[i * pl + nx + 1] : 0.;
  }
  __syncthreads();  // all[] initialised
#pragma unroll
  for (int i = 0; i < kClsLayers; i++) {
    const double a = q[i][0];
    const bool c = !in || (q[i][1] == a && q[i][2] == a && q[i][3] == a && q[i + 1][0] == a &&
                           q[i + 1][1] == a && q[i + 1][2] == a && q[i + 1][3] == a);
    if (!__all_sync(0xffffffffu, c) && threadIdx.x == 0) all[i] = 0;
  }
  __syncthreads();
  if (tid < kClsLayers && k0 + tid < nez)
    cls[(int64_t)(blockIdx.y * gridDim.x + blockIdx.x) * nez + k0 + tid] = all[tid] ? 1 : 0;
}

// Exclusive prefix sum of a[0, n) in shared memory over the whole block (blockDim.x a
// multiple of 32, at most 1024); returns the total.  wsum: 32 ints of shared scratch.
__device__ int block_scan_excl(int* a, int n, int* wsum) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b0 = min((int)threadIdx.x * per, n), b1 = min(b0 + per, n);
  int sum = 0;
  for (int i = b0; i < b1; i++) sum += a[i];
  int x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nw ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  int run = x - sum + (warp ? wsum[warp - 1] : 0);
  const int total = wsum[nw - 1];
  for (int i = b0; i < b1; i++) {
    const int t = a[i];
    a[i] = run;
    run += t;
  }
  __syncthreads();  // wsum is reused by the next scan
  return total;
}

// Unit type of node plane z of a tile column from its layer flags f[0, nz - 1):
// 0 when the element layers below and above are constant (or absent), else 1.
__device__ __forceinline__ int unit_type(const uint8_t* f, int z, int nez) {
  const bool below = z == 0 || f[z - 1], above = z == nez || f[z];
  return below && above ? 0 : 1;
}

// One block of 1024 threads builds both unit lists of a plan from its layer flags:
// per tile column (one thread each) the runs of equal unit type up its nz planes,
// counted, offset by prefix sums over the columns in tile order, written; then, per
// list l and block b of its wave of ncta_l blocks, the run holding the list's unit
// U b / ncta_l (binary search on the runs' unit offsets).
__global__ void __launch_bounds__(1024) unit_lists_kernel(const uint8_t* __restrict__ cls, int nz,
                                                          int ncol, int ncta0, int ncta1, int4* __restrict__ runs0,
                                                          int4* __restrict__ runs1, int* __restrict__ start0,
                                                          int* __restrict__ start1, int* __restrict__ total) {
  extern __shared__ int sh[];  // [4][ncol] counts, then 32 ints of scan scratch
  int* cnt = sh;
  int* wsum = sh + 4 * ncol;
  const int nez = nz - 1;
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
    const uint8_t* f = cls + (int64_t)c * nez;
    int nr[2] = {0, 0}, nu[2] = {0, 0}, prev = -1;
    for (int z = 0; z < nz; z++) {
      const int t = unit_type(f, z, nez);
      nu[t]++;
      if (t != prev) nr[t]++;
      prev = t;
    }
    cnt[c] = nr[0];
    cnt[ncol + c] = nr[1];
    cnt[2 * ncol + c] = nu[0];
    cnt[3 * ncol + c] = nu[1];
  }
  __syncthreads();
  int tot[4];
#pragma unroll
  for (int a = 0; a < 4; a++) tot[a] = block_scan_excl(cnt + a * ncol, ncol, wsum);
  int4* runs[2] = {runs0, runs1};
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
    const uint8_t* f = cls + (int64_t)c * nez;
    int r[2] = {cnt[c], cnt[ncol + c]}, u[2] = {cnt[2 * ncol + c], cnt[3 * ncol + c]};
    int z0 = 0, t0 = unit_type(f, 0, nez);
    for (int z = 1; z <= nz; z++) {
      const int t = z < nz ? unit_type(f, z, nez) : -1;
      if (t != t0) {
        runs[t0][r[t0]++] = make_int4(c, z0, z, u[t0]);
        u[t0] += z - z0;
        z0 = z;
        t0 = t;
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < ncta0 + ncta1; i += blockDim.x) {
    const int l = i < ncta0 ? 0 : 1, b = l ? i - ncta0 : i, ncta = l ? ncta1 : ncta0, nrun = tot[l];
    const int64_t ub = (int64_t)tot[2 + l] * b / ncta;
    int lo = 0, hi = nrun - 1;
    while (lo < hi) {  // the last run whose first unit is <= ub
      const int mid = (lo + hi + 1) / 2;
      if (runs[l][mid].w <= ub) lo = mid; else hi = mid - 1;
    }
    (l ? start1 : start0)[b] = nrun > 0 ? lo : 0;
  }
  if (threadIdx.x == 0) {
    total[0] = tot[2];
    total[1] = tot[3];
  }
}

constexpr int kMaxListCols = 2048;  // tile columns the one-block list builder takes
// Grids below this many (tile, plane) units keep the plain split: there the general
// wave's latency (about one segment) and the list build cost more than the fixed-weight
// kernel saves.  Measured on the penny field, split against plain, us per apply FP64 /
// FP32: 41^3 35.8 / 29.7 against 25.7 / 23.6; 65^3 44.1 / 35.9 against 44.0 / 29.5;
// 81^3 54.3 / 46.0 against 60.4 / 42.1; 97^3 64.5 / 56.3 against 72.7 / 52.2; 113^3
// 93.3 / 72.8 against 109.6 / 74.8; 161^3 189.4 / 140.3 against 247.0 / 154.7.
#ifndef VFGPU_U64_LISTS_MIN_UNITS
#define VFGPU_U64_LISTS_MIN_UNITS 2000
#endif
#ifndef VFGPU_U32_LISTS_MIN_UNITS
#define VFGPU_U32_LISTS_MIN_UNITS 6000
#endif

bool unit_lists_pay(const TilePlan& p, int nz, int prec_bytes) {
  const int64_t min_units = prec_bytes == 8 ? VFGPU_U64_LISTS_MIN_UNITS : VFGPU_U32_LISTS_MIN_UNITS;
  return (int64_t)p.ntx * p.nty * nz >= min_units;
}

size_t unit_lists_bytes(const TilePlan& p, int nz) {
  const int64_t ncol = (int64_t)p.ntx * p.nty;
  if (nz < 2 || ncol > kMaxListCols) return 0;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  return up(ncol * (nz - 1)) + 2 * up(ncol * nz * sizeof(int4)) + up(p.ncta0 * sizeof(int)) +
         up(p.ncta * sizeof(int)) + up(2 * sizeof(int));
}

UnitLists unit_lists_carve(void* base, const TilePlan& p, int nz) {
  UnitLists L;
  if (!base || !unit_lists_bytes(p, nz)) return L;
  const size_t ncol = (size_t)p.ntx * p.nty;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  char* q = static_cast<char*>(base);
  L.cls = reinterpret_cast<uint8_t*>(q);
  q += up(ncol * (nz - 1));
  for (int l = 0; l < 2; l++) {
    L.runs[l] = reinterpret_cast<int4*>(q);
    q += up(ncol * nz * sizeof(int4));
  }
  for (int l = 0; l < 2; l++) {
    L.start[l] = reinterpret_cast<int*>(q);
    q += up((l ? p.ncta : p.ncta0) * sizeof(int));
  }
  L.total = reinterpret_cast<int*>(q);
  return L;
}

template <int TY>
static cudaError_t classify(const double* v, uint8_t* cls, int nx, int ny, int nz, const TilePlan& p,
                            cudaStream_t s) {
  const int runs = (nz - 1 + kClsLayers - 1) / kClsLayers;
  if (runs > 65535 || p.nty > 65535) return cudaErrorInvalidValue;
  u_classify_kernel<TY><<<dim3(p.ntx, p.nty, runs), dim3(32, TY), 0, s>>>(v, cls, nx, ny, nz - 1);
  return cudaGetLastError();
}

cudaError_t build_unit_lists(const double* v, int nx, int ny, int nz, const TilePlan& p,
                             const UnitLists& L, cudaStream_t s) {
  if (!L.cls) return cudaSuccess;
  cudaError_t e;
  switch (p.ty) {
    case 4: e = classify<4>(v, L.cls, nx, ny, nz, p, s); break;
    case 8: e = classify<8>(v, L.cls, nx, ny, nz, p, s); break;
    case 16: e = classify<16>(v, L.cls, nx, ny, nz, p, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  const int ncol = p.ntx * p.nty;
  unit_lists_kernel<<<1, 1024, (4 * ncol + 32) * sizeof(int), s>>>(
      L.cls, nz, ncol, p.ncta0, p.ncta, L.runs[0], L.runs[1], L.start[0], L.start[1], L.total);
  return cudaGetLastError();
}

TilePlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms) {
  TilePlan p = tile_plan(nx, ny, nz, prec_bytes == 8 ? U64_TY : U32_TY, 3,
                         prec_bytes == 8 ? U64_MINB : U32_MINB, num_sms);
  const TilePlan q = tile_plan(nx, ny, nz, p.ty, 3, prec_bytes == 8 ? U64C_MINB : U32C_MINB, num_sms);
  p.ncta0 = q.ncta;
  return p;
}
TilePlan v_plan(int nx, int ny, int nz, int prec_bytes, int num_sms) {
  return tile_plan(nx, ny, nz, V_TY, 1, prec_bytes == 8 ? V64_MINB : V32_MINB, num_sms);
}

// The 1-D tensor maps of x (3N values) and v (N) that the fixed-weight wave copies its node
// planes with (PlaneBox boxes, zeros beyond the ends); false where they cannot be made:
// a pointer not 16-byte aligned, 3N past the 32-bit coordinates, no encoder.
template <typename T> static bool u_plane_maps(UApplyArgs<T>& A) {
  const int64_t N = (int64_t)A.nx * A.ny * A.nz;
  const TensorEncode encode = tensor_encode();
  if (!encode || 3 * N >= (int64_t)INT32_MAX || ((uintptr_t)A.x & 15) || ((uintptr_t)A.v & 15)) return false;
  const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dx[1] = {(cuuint64_t)(3 * N)}, dv[1] = {(cuuint64_t)N}, none[1] = {0};
  const cuuint32_t bx[1] = {(cuuint32_t)PlaneBox<T>::XBOX}, bv[1] = {(cuuint32_t)PlaneBox<T>::VBOX}, es[1] = {1};
  const CUresult r1 = encode(&A.xmap, dt, 1, const_cast<T*>(A.x), dx, none, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  const CUresult r2 = encode(&A.vmap, dt, 1, const_cast<T*>(A.v), dv, none, bv, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r1 == CUDA_SUCCESS && r2 == CUDA_SUCCESS;
}

// A split launch's operands (with the VFGPU_U_PLANES_TMA build option, the plane maps), or
// false: then the apply runs one wave, with the second wave's x.y partials zeroed for a
// caller that counts them.
template <typename T> static bool split_args(const UApplyArgs<T>& A, const TilePlan& p, UApplyArgs<T>& B,
                                             cudaStream_t s) {
  B = A;
  if (!VFGPU_U_PLANES_TMA || u_plane_maps(B)) return true;
  if (A.dot) cudaMemsetAsync(A.dot + p.ncta + seam_blocks(p, A.nx, A.ny, A.nz), 0, p.ncta0 * sizeof(double), s);
  return false;
}

template <>
cudaError_t launch_u_apply<double>(const UApplyArgs<double>& A, const TilePlan& p,
                                   const LayerTable& L, cudaStream_t s) {
  if (A.cflag) return launch_tile_apply<UOpNC<double>, U64_TY, 1>(A, p, L, s);
  UApplyArgs<double> B;
  if (A.ur[0] && A.ur[1] && split_args(A, p, B, s)) {
    if (cubic(A))
      return launch_tile_apply_split<UOpConst<double, true>, UOp<double, true>, U64_TY, U64C_MINB, U64_MINB>(
          B, p, L, s);
    return launch_tile_apply_split<UOpConst<double>, UOp<double>, U64_TY, U64C_MINB, U64_MINB>(B, p, L, s);
  }
  if (cubic(A)) return launch_tile_apply<UOp<double, true>, U64_TY, U64_MINB>(A, p, L, s);
  return launch_tile_apply<UOp<double>, U64_TY, U64_MINB>(A, p, L, s);
}
template <>
cudaError_t launch_u_apply<float>(const UApplyArgs<float>& A, const TilePlan& p,
                                  const LayerTable& L, cudaStream_t s) {
  // NOCOMPRESSION needs the scalar layout: its plan is the FP32 plan only with the
  // scalar tile (the packed build option keeps the plain operator packed)
  if (A.cflag) return launch_tile_apply<UOpNC<float>, U_TY, 2>(A, p, L, s);
  if constexpr (!kU32Packed) {
    UApplyArgs<float> B;
    if (A.ur[0] && A.ur[1] && split_args(A, p, B, s)) {
      if (cubic(A))
        return launch_tile_apply_split<U32COpC, U32OpC, U32_TY, U32C_MINB, U32_MINB>(B, p, L, s);
      return launch_tile_apply_split<U32COp, U32Op, U32_TY, U32C_MINB, U32_MINB>(B, p, L, s);
    }
  }
  if (cubic(A)) return launch_tile_apply<U32OpC, U32_TY, U32_MINB>(A, p, L, s);
  return launch_tile_apply<U32Op, U32_TY, U32_MINB>(A, p, L, s);
}
template <>
cudaError_t launch_v_apply<double>(const VApplyArgs<double>& A, const TilePlan& p,
                                   const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<VOp<double>, V_TY, V64_MINB>(A, p, L, s);
}
template <>
cudaError_t launch_v_apply<float>(const VApplyArgs<float>& A, const TilePlan& p,
                                  const LayerTable& L, cudaStream_t s) {
  return launch_tile_apply<VOp<float>, V_TY, V32_MINB>(A, p, L, s);
}

}  // namespace vfgpu

extern "C" int vfgpu_wait_selftest(long long cycles, int complete, int* timed_out) {
  if (!timed_out || cycles < 0 || cycles > 4000000000ll) return -1;
  return vfgpu::wait_selftest(cycles, complete ? 1 : 0, timed_out) == cudaSuccess ? 0 : -2;
}
