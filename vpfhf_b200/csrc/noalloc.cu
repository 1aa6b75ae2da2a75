// noalloc.cu -- a U-operator apply that performs no device allocation.
//
// Who needs it: code that must not call cudaMalloc while it runs -- for example
// a matrix-shell callback inside an external Krylov solver whose host program
// owns every device buffer (fixed memory budget, pool allocator), or a hot loop
// that cannot afford cudaMalloc's implicit device-wide synchronisation.  Such a
// caller cannot create a vfgpu_ctx (vfgpu_create allocates the fields and work
// space), so this entry point takes every array from the caller and keeps its
// only scratch -- the seam partial sums of the tiled apply -- in one fixed,
// file-scope device array.  That array is part of the loaded module: every GPU
// that loads the library holds its 32 MiB until the process exits.
#include <cstring>

#include "abi_util.h"
#include "kernels.h"

namespace {

constexpr size_t kScratchDoubles = VFGPU_NOALLOC_SCRATCH_DOUBLES;

// Seam partials of the last call; every slot the fix-up kernel reads is written
// earlier in the same call, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of the scratch array in the current device's context.  Looked up on
// every call (a host-side table lookup, no device work): the host-side symbol is not
// a device address, and a cached address would go stale when the context is rebuilt
// (cudaDeviceReset, or another primary context after a reset elsewhere in the process).
int scratch_address(double** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return vfgpu::cuda_fail(e, "vfgpu_u_apply_noalloc: cudaGetSymbolAddress");
  *out = static_cast<double*>(p);
  return VFGPU_OK;
}

}  // namespace

extern "C" int vfgpu_u_apply_noalloc(const vfgpu_grid* g, const vfgpu_matprop* mp, double eta,
                                     const double* v, const unsigned char* bcbits, const double* x,
                                     double* y, void* stream) {
  using namespace vfgpu;
  if (!g || !mp || !v || !x || !y)
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_noalloc: null argument");
  if (g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->lx > 0) || !(g->ly > 0) || !(g->lz > 0))
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_noalloc: bad grid");
  if ((int64_t)g->nx * g->ny * g->nz * 3 >= (int64_t)1 << 31)
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_noalloc: grid too large for int32 indexing");
  if (!(mp->E > 0) || !(mp->nu > -1 && mp->nu < 0.5) || !(eta >= 0))
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_noalloc: need E > 0, -1 < nu < 0.5, eta >= 0");
  if (!is_device_ptr(v) || !is_device_ptr(x) || !is_device_ptr(y) ||
      (bcbits && !is_device_ptr(bcbits)))
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_noalloc: v, x, y, bcbits must be device pointers");
  int dev = 0, nsm = 148;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_noalloc: cudaGetDevice");
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const TilePlan p = u_plan(g->nx, g->ny, g->nz, 8, nsm);
  if (p.seamX + p.seamY > kScratchDoubles)
    return fail(VFGPU_ERR_INVALID,
                "vfgpu_u_apply_noalloc: grid %dx%dx%d needs %zu scratch doubles, the fixed "
                "scratch holds %zu (use vfgpu_u_apply with a vfgpu_ctx)",
                g->nx, g->ny, g->nz, p.seamX + p.seamY, kScratchDoubles);
  {
    // out of place only: the tiles read x planes and Dirichlet rows copy x while other
    // blocks write y
    const uintptr_t n3 = (uintptr_t)g->nx * g->ny * g->nz * 3 * sizeof(double);
    const uintptr_t xb = reinterpret_cast<uintptr_t>(x), yb = reinterpret_cast<uintptr_t>(y);
    if (xb < yb + n3 && yb < xb + n3)
      return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_noalloc: x and y overlap (the apply is out of place)");
  }
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  // the kernels' shared-memory opt-in, under the same lock vfgpu_create takes
  e = apply_kernel_attributes();
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_noalloc: kernel attributes");
  LayerTable L{};
  L.lambda[0] = mp->E * mp->nu / (1. + mp->nu) / (1. - 2. * mp->nu);  // VFCommon.c:584
  L.mu[0] = mp->E / (1. + mp->nu) * .5;                                // VFCommon.c:585
  UApplyArgs<double> A{};
  A.x = x;
  A.v = v;
  A.y = y;
  A.bc = bcbits;
  A.seamX = scratch;
  A.seamY = scratch + p.seamX;
  A.nx = g->nx;
  A.ny = g->ny;
  A.nz = g->nz;
  const double hx = g->lx / (g->nx - 1.), hy = g->ly / (g->ny - 1.), hz = g->lz / (g->nz - 1.);
  A.ihx = 1.0 / hx;
  A.ihy = 1.0 / hy;
  A.ihz = 1.0 / hz;
  A.vol = hx * hy * hz;
  A.eta = eta;
  e = launch_u_apply<double>(A, p, L, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_noalloc");
  return VFGPU_OK;
}
