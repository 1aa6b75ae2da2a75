// abi_util.h -- helpers shared by the C-ABI translation units.
#pragma once

#include <functional>

#include "ctx.h"

namespace vfgpu {
// The StepU preconditioner a solve option resolves to on an nx x ny x nz grid
// (VFGPU_PC_AUTO: multigrid where some axis has VFGPU_PC_AUTO_MG_NODES nodes or more).
inline int resolve_pc(int pc, int nx, int ny, int nz) {
  if (pc != VFGPU_PC_AUTO) return pc;
  const int m = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  return m >= VFGPU_PC_AUTO_MG_NODES ? VFGPU_PC_MG : VFGPU_PC_JACOBI;
}
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
bool is_device_ptr(const void* p);
cudaError_t copy_in(vfgpu_ctx* c, double* dst, const double* src, int64_t n);
cudaError_t copy_out(vfgpu_ctx* c, double* dst, const double* src, int64_t n);
int ensure_v32(vfgpu_ctx* c);
void free_solver(vfgpu_ctx* c);
int upload_params(vfgpu_ctx* c);
// NOCOMPRESSION: recompute the per-cell compression bits from displacement u (device).
cudaError_t nc_flags(vfgpu_ctx* c, const double* u);
// Geometric multigrid preconditioned CG of the U Jacobian (mg.cu): x = K^-1 b, FP64
// Krylov vectors, V-cycle in FP32 (fp32) or FP64, with the stopping test of the
// Jacobi PCG (dinv0 = FP64 inverse diagonal; dinv0_32 its FP32 copy for fp32).
// reuse: the operator is unchanged since the last call (keeps the level set-up).
int run_mgcg(vfgpu_ctx* c, bool fp32, const double* b, double* x, double* r, double* p, double* w,
             const double* dinv0, const float* dinv0_32, bool reuse, double rtol, double atol,
             double dtol, int maxit, int* its, int* reason, int* levels);
// Graph of one call site's launch sequence, captured on first use and re-captured when
// ctx->gen moves on (null: capture failed, run the body directly).
cudaGraphExec_t ctx_graph(vfgpu_ctx* c, int kind, int batch,
                          const std::function<cudaError_t()>& body);
void free_mg(vfgpu_ctx* c);
// Device bytes of the multigrid hierarchy of a grid in V-cycle precision `bytes` (4 or 8),
// a per-cell modulus included; 0 when the grid has no coarse level.
long long mg_memory_bytes(int nx, int ny, int nz, int bytes);
template <typename T>
UApplyArgs<T> u_args(vfgpu_ctx* c, const T* x, const T* v, T* y, T* seam, const TilePlan& p);
// Rebuilds the U unit lists (which u_args passes) from the FP64 v on the ctx stream if
// v changed since they were built: every entry that applies U calls it first.
cudaError_t u_lists_refresh(vfgpu_ctx* c);
// Whether the ctx's U applies in this precision (8 or 4 bytes) take the unit lists (and
// write the second wave's x.y partials).
bool u_lists_on(const vfgpu_ctx* c, int prec_bytes);
}  // namespace vfgpu
