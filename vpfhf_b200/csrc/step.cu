// step.cu -- the U and V solves (VF_StepU / VF_StepV), the time-step preparation
// and the energy / crack-opening reductions behind the C ABI.
#include <chrono>
#include <cmath>
#include <cstring>

#include "abi_util.h"
#include "solver.h"
#include "vec.h"

using namespace vfgpu;

namespace vfgpu {

void free_solver(vfgpu_ctx* c) {
  for (auto& p : c->p64) cudaFree(p), p = nullptr;
  for (auto& p : c->p32) cudaFree(p), p = nullptr;
  cudaFree(c->coef64);
  cudaFree(c->coef32);
  cudaFree(c->vmask);
  cudaFree(c->d_cg);
  cudaFree(c->d_red);
  cudaFree(c->d_out);
  if (c->h_cg) cudaFreeHost(c->h_cg);
  if (c->h_out) cudaFreeHost(c->h_out);
  c->coef64 = nullptr;
  c->coef32 = nullptr;
  c->vmask = nullptr;
  c->d_cg = nullptr;
  c->d_red = nullptr;
  c->d_out = nullptr;
  c->h_cg = nullptr;
  c->h_out = nullptr;
  c->have_solver = false;
}

static int solve_buffers(vfgpu_ctx* c) {
  if (c->have_solver) return VFGPU_OK;
  cudaError_t e = cudaSuccess;
  // 3N values plus slack, so that three N-vectors carved at 16-byte aligned offsets fit
  const size_t n3 = 3 * (size_t)c->N + kPoolSlack;
  for (auto& p : c->p64)
    if (e == cudaSuccess) e = cudaMalloc((void**)&p, n3 * sizeof(double));
  for (auto& p : c->p32)
    if (e == cudaSuccess) e = cudaMalloc((void**)&p, n3 * sizeof(float));
  const size_t ncoef = (size_t)vcoef_size(c->nx - 1, c->ny - 1, c->nz - 1);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->coef64, ncoef * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->coef32, ncoef * sizeof(float));
  // row padding is copied but never used; keep it defined
  if (e == cudaSuccess) e = cudaMemsetAsync(c->coef64, 0, ncoef * sizeof(double), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->coef32, 0, ncoef * sizeof(float), c->stream);
  if (e == cudaSuccess)
    e = vcoef_tensor_map(&c->vmap64, c->coef64, 8, c->nx - 1, c->ny - 1, c->nz - 1);
  if (e == cudaSuccess)
    e = vcoef_tensor_map(&c->vmap32, c->coef32, 4, c->nx - 1, c->ny - 1, c->nz - 1);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->vmask, (size_t)c->N);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_cg, sizeof(CGState));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&c->d_red, (size_t)(RED_BLOCKS + energy_blocks()) * 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_out, 16 * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_cg, sizeof(CGState));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_out, 16 * sizeof(double));
  etab_host(c->hx, c->hy, c->hz, &c->h_tab);
  if (e != cudaSuccess) {
    free_solver(c);
    return cuda_fail(e, "solver work space");
  }
  c->have_solver = true;
  return VFGPU_OK;
}

static ElemArgs elem_args(vfgpu_ctx* c) {
  ElemArgs E{};
  E.tab = c->h_tab;
  E.nx = c->nx;
  E.ny = c->ny;
  E.nz = c->nz;
  E.elayer = c->d_elayer;
  E.cellE = c->d_cellE;
  E.L = c->layers;
  E.eta = c->vf.eta;
  E.epsilon = c->vf.epsilon;
  E.atcv = c->vf.atnum == 1 ? 2. / 3. : .5;  // VFCommon.c:482-492
  E.atnum = c->vf.atnum;
  E.hasCrackPressure = c->vf.hasCrackPressure;
  E.unilateral = c->unilateral;
  E.hx = c->hx;
  E.hy = c->hy;
  E.hz = c->hz;
  return E;
}

cudaError_t nc_flags(vfgpu_ctx* c, const double* u) {
  if (!c->unilateral) return cudaSuccess;
  if (solve_buffers(c) != VFGPU_OK) return cudaErrorMemoryAllocation;
  return launch_nc_flags(elem_args(c), u, c->d_cflag, c->stream);
}

static InsituArgs insitu_args(const vfgpu_ctx* c) {
  InsituArgs A{};
  A.nx = c->nx;
  A.ny = c->ny;
  A.nz = c->nz;
  A.hx = c->hx;
  A.hy = c->hy;
  A.hz = c->hz;
  A.lz = c->lz;
  for (int i = 0; i < 6; i++) {
    A.smin[i] = c->insitu_min[i];
    A.smax[i] = c->insitu_max[i];
  }
  for (int f = 0; f < 6; f++)
    for (int comp = 0; comp < 3; comp++) A.freec[f][comp] = c->bcU[comp].face[f] == VFGPU_BC_NONE;
  return A;
}

// f (3N) = the U load of VF_UResidual: thermo-poro, crack pressure and in-situ tractions;
// u0: the displacement that fixes the NOCOMPRESSION sign pattern of the thermo-poro term.
static cudaError_t u_load(vfgpu_ctx* c, const ElemArgs& E, double* f, const double* u0) {
  cudaError_t e = launch_u_rhs(E, c->f[VFGPU_FIELD_V], c->f[VFGPU_FIELD_THETA],
                               c->f[VFGPU_FIELD_THETAREF], c->f[VFGPU_FIELD_PRESSURE], f, c->stream,
                               u0);
  if (e == cudaSuccess && c->has_insitu) e = launch_insitu_load(insitu_args(c), f, c->stream);
  return e;
}

template <typename T>
static VApplyArgs<T> v_args(vfgpu_ctx* c, const T* x, T* y, const uint8_t* mask,
                            const CUtensorMap& cmap, T* seam, const TilePlan& p) {
  VApplyArgs<T> A{};
  A.cmap = cmap;
  A.cerr = c->d_cerr;
  A.x = x;
  A.y = y;
  A.mask = mask;
  A.elayer = c->d_elayer;
  A.seamX = seam;
  A.seamY = seam + p.seamX;
  A.nx = c->nx;
  A.ny = c->ny;
  A.nz = c->nz;
  A.ihx = T(1.0 / c->hx);
  A.ihy = T(1.0 / c->hy);
  A.ihz = T(1.0 / c->hz);
  A.vol = T(c->hx * c->hy * c->hz);
  A.P = c->d_params;
  return A;
}

// VFGPU_ERR_CUDA when a V apply gave up waiting for its coefficient copies (the
// flag is cleared for the next solve).
static int check_cell_copies(vfgpu_ctx* c) {
  unsigned flag = 0;
  cudaError_t e = cudaMemcpyAsync(&flag, c->d_cerr, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "V apply");
  if (!flag) return VFGPU_OK;
  cudaMemsetAsync(c->d_cerr, 0, sizeof(unsigned), c->stream);
  return fail(VFGPU_ERR_CUDA, "operator apply: a tensor copy (V coefficients or U node planes) did not "
                              "complete in time");
}

// Reads n doubles of d_out into h_out (synchronising the stream).
static cudaError_t fetch(vfgpu_ctx* c, int n) {
  cudaError_t e = cudaMemcpyAsync(c->h_out, c->d_out, n * sizeof(double), cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e;
}

static double dot_host(vfgpu_ctx* c, const double* a, const double* b, int64_t n, cudaError_t& e) {
  const double* pa[1] = {a};
  const double* pb[1] = {b};
  if (e == cudaSuccess) e = dev_dots(pa, pb, 1, n, c->d_red, c->d_out, c->stream);
  if (e == cudaSuccess) e = fetch(c, 1);
  return e == cudaSuccess ? c->h_out[0] : NAN;
}

using clk = std::chrono::steady_clock;

struct Watch {
  clk::time_point t0 = clk::now();
  double limit = 0;
  bool expired() const {
    return limit > 0 && std::chrono::duration<double>(clk::now() - t0).count() > limit;
  }
  double seconds() const { return std::chrono::duration<double>(clk::now() - t0).count(); }
};

// PCG with device-side convergence: queues batches of iterations (every kernel of a
// converged solve is a no-op), checks the flag between batches.
// Graph of `batch` CG iterations for call site `kind`, captured on first use (the
// kernels' pointers are fixed per call site; see vfgpu_ctx::Graph).
template <class Body>
static cudaGraphExec_t cg_graph(vfgpu_ctx* c, int kind, int batch, Body body) {
  for (auto& g : c->graphs)
    if (g.kind == kind && g.batch == batch) {
      if (g.gen == c->gen) return g.exec;
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  const cudaError_t eb = body();
  const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
  if (eb != cudaSuccess || ec != cudaSuccess || !graph ||
      cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return nullptr;
  }
  cudaGraphDestroy(graph);
  bool stored = false;
  for (auto& g : c->graphs)
    if (g.kind == kind && g.batch == batch) {
      g.exec = exec;
      g.gen = c->gen;
      stored = true;
    }
  if (!stored) c->graphs.push_back({kind, batch, c->gen, exec});
  return exec;
}

cudaGraphExec_t ctx_graph(vfgpu_ctx* c, int kind, int batch,
                          const std::function<cudaError_t()>& body) {
  return cg_graph(c, kind, batch, body);
}

template <typename T, class Apply>
static int run_cg(vfgpu_ctx* c, int kind, const CGVecs<T>& v, Apply apply, double rtol,
                  double atol, double dtol, int maxit, const Watch& w, int* its, int* reason,
                  bool* timeout) {
  cudaError_t e = cg_init<T>(v, c->d_cg, c->d_red, rtol, atol, dtol, maxit, c->stream);
  // Batches of iterations are queued without a host round trip; a converged CG turns
  // the rest of a batch into no-ops (skip flag), so the batch sizes do not change the
  // result.  The first batch is the largest power of two (4..64) not above the call
  // site's last iteration count, and is queued before the first host check.
  int batch = 4;
  while (batch < 64 && 2 * batch <= c->cg_last_its[kind & 7]) batch *= 2;
  bool first = true;
  *timeout = false;
  auto body = [&](int nb) {
    cudaError_t eb = cudaSuccess;
    for (int b = 0; b < nb && eb == cudaSuccess; b++) {
      eb = apply(v.p, v.w, &c->d_cg->done, const_cast<double*>(v.dotp));
      if (eb == cudaSuccess) eb = cg_after_apply<T>(v, c->d_cg, c->d_red, c->stream);
    }
    return eb;
  };
  while (e == cudaSuccess) {
    if (!first) {
      e = cudaMemcpyAsync(c->h_cg, c->d_cg, sizeof(CGState), cudaMemcpyDeviceToHost, c->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
      if (e != cudaSuccess || c->h_cg->done) break;
      if (w.expired()) {
        *timeout = true;
        break;
      }
      batch = std::min(batch * 2, 64);
    }
    first = false;
    cudaGraphExec_t g = c->use_graphs ? cg_graph(c, kind, batch, [&] { return body(batch); }) : nullptr;
    e = g ? cudaGraphLaunch(g, c->stream) : body(batch);
  }
  // the step of the iteration that stopped the solve has not reached x yet
  if (e == cudaSuccess) e = cg_finish_x<T>(v, c->d_cg, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "CG");
  *its = c->h_cg->its;
  *reason = c->h_cg->reason;
  c->cg_last_its[kind & 7] = *its;
  return VFGPU_OK;
}

// ---------------------------------------------------------------------------- U
// dot: if non-null the apply also writes the block partials of x.y there (the CG's p.w)
static cudaError_t u_apply64(vfgpu_ctx* c, const double* x, double* y, const int* skip,
                             double* dot = nullptr) {
  UApplyArgs<double> A = u_args<double>(c, x, c->f[VFGPU_FIELD_V], y, c->seam64, c->plan64);
  A.skip = skip;
  A.dot = dot;
  return launch_u_apply<double>(A, c->plan64, c->layers, c->stream);
}
static cudaError_t u_apply32(vfgpu_ctx* c, const float* x, float* y, const int* skip,
                             double* dot = nullptr) {
  UApplyArgs<float> A = u_args<float>(c, x, c->V32, y, c->seam32, c->plan32);
  A.skip = skip;
  A.dot = dot;
  return launch_u_apply<float>(A, c->plan32, c->layers, c->stream);
}
static int dots_of(const vfgpu_ctx* c, const TilePlan& p) { return tile_dot_count(p, c->nx, c->ny, c->nz); }
// The U applies of a split launch (unit lists) write a second wave's partials.
static int u_dots_of(const vfgpu_ctx* c, const TilePlan& p, int prec_bytes) {
  return dots_of(c, p) + (u_lists_on(c, prec_bytes) ? p.ncta0 : 0);
}

// Which CG call sites let the operator apply accumulate p.w (bit k-1 for call site k:
// 1 U FP64, 2 U FP32, 3 V FP64, 4 V FP32); the others use a separate p.w pass.  U in
// both precisions and V in FP64: the 129^3 mixed StepU measured 37.07 ms with the FP32
// U apply accumulating p.w (the packed FP32 fixed-weight wave has the registers for it)
// against 37.78 ms with the separate pass; with the earlier single-wave FP32 kernel the
// accumulator spilled (U FP32 0.064 s fused-off against 0.066 s fused-on; FP64 U 0.0957 s
// fused, 0.0972 s separate).  V FP32 fused as well measured 6.44 against 6.50 ms per
// mixed StepV: not taken.
#ifndef VFGPU_FUSE_DOT_MASK
#define VFGPU_FUSE_DOT_MASK 7
#endif
static double* dot_buf(vfgpu_ctx* c, int kind) {
  return ((VFGPU_FUSE_DOT_MASK >> (kind - 1)) & 1) ? c->d_dot : nullptr;
}

// F = K(V) U - f, Dirichlet rows U - ubc (VF_UResidual, VFMech.c:1456-1887).
static cudaError_t u_residual(vfgpu_ctx* c, const double* u, const double* f, double* tmp,
                              double* F) {
  cudaError_t e = u_apply64(c, u, tmp, nullptr);
  if (e == cudaSuccess)
    e = dev_u_residual(tmp, f, u, c->bcU_kind, c->f[VFGPU_FIELD_BCU], F, 3 * c->N, c->stream);
  return e;
}

}  // namespace vfgpu

extern "C" {

void vfgpu_default_solve_opts(vfgpu_solve_opts* o) {
  if (!o) return;
  // VFCommon.c:1024 (SNES atol = rtol = 1e-8) and :1039 (KSP rtol 1e-8, atol 1e-10)
  o->precision = VFGPU_FP64;
  o->ksp_rtol = 1e-8;
  o->ksp_atol = 1e-10;
  o->ksp_dtol = 1e5;
  o->ksp_maxit = 10000;
  o->snes_rtol = 1e-8;
  o->snes_atol = 1e-8;
  o->snes_stol = 1e-8;
  o->snes_maxit = 50;
  o->inner_rtol = 1e-4;
  o->max_refine = 12;
  o->time_limit = 0.;
  o->pc = VFGPU_PC_JACOBI;
}

int vfgpu_step_u(vfgpu_ctx* c, const vfgpu_solve_opts* o_, vfgpu_solve_stats* st) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_step_u: null ctx");
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "vfgpu_step_u: material not set");
  vfgpu_solve_opts o;
  if (o_) o = *o_; else vfgpu_default_solve_opts(&o);
  if (o.precision != VFGPU_FP64 && o.precision != VFGPU_MIXED)
    return fail(VFGPU_ERR_INVALID, "vfgpu_step_u: bad precision");
  if (o.pc != VFGPU_PC_JACOBI && o.pc != VFGPU_PC_MG && o.pc != VFGPU_PC_AUTO)
    return fail(VFGPU_ERR_INVALID, "vfgpu_step_u: bad preconditioner");
  o.pc = resolve_pc(o.pc, c->nx, c->ny, c->nz);
  vfgpu_solve_stats S{};
  cudaSetDevice(c->dev);
  int rc = solve_buffers(c);
  if (rc) return rc;
  Watch w;
  w.limit = o.time_limit;
  const int64_t n3 = 3 * c->N;
  double *f = c->p64[0], *dinv = c->p64[1], *F = c->p64[2], *Y = c->p64[3], *JY = c->p64[4];
  double *R = c->p64[5], *P = c->p64[6], *W = c->p64[7];
  double* U = c->f[VFGPU_FIELD_U];
  const bool mixed = o.precision == VFGPU_MIXED;
  ElemArgs E = elem_args(c);
  const bool nc = c->unilateral != 0;
  cudaError_t e = u_lists_refresh(c);  // v is fixed for the whole solve
  if (e == cudaSuccess) e = nc_flags(c, U);
  if (e == cudaSuccess) e = u_load(c, E, f, U);
  if (e == cudaSuccess) e = launch_u_diag(E, c->f[VFGPU_FIELD_V], c->bcU_bits, JY, c->stream, U);
  if (e == cudaSuccess) e = dev_inv(JY, dinv, mixed ? c->p32[4] : nullptr, n3, c->stream);
  if (mixed && e == cudaSuccess) {
    rc = ensure_v32(c);
    if (rc) return rc;
  }
  if (e == cudaSuccess) e = u_residual(c, U, f, JY, F);
  double fnorm = dot_host(c, F, F, n3, e);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
  fnorm = sqrt(fnorm);
  S.fnorm0 = fnorm;
  const double ttol = o.snes_rtol * fnorm;
  int reason = 0;
  if (fnorm < o.snes_atol) reason = 2;  // SNES_CONVERGED_FNORM_ABS
  auto apply64 = [&](const double* x, double* y, const int* skip, double* dot) {
    return u_apply64(c, x, y, skip, dot);
  };
  auto apply32 = [&](const float* x, float* y, const int* skip, double* dot) {
    return u_apply32(c, x, y, skip, dot);
  };
  // NOCOMPRESSION: F(X) = K(V; X) X - f(X) with the sign pattern of X (flags left at X)
  auto nc_residual = [&](const double* X, double* Fout) {
    cudaError_t ee = nc_flags(c, X);
    if (ee == cudaSuccess) ee = u_load(c, E, f, X);
    if (ee == cudaSuccess) ee = u_residual(c, X, f, JY, Fout);
    return ee;
  };
  for (int it = 0; !reason && it < o.snes_maxit; it++) {
    int kits = 0, kreason = 0;
    bool tmo = false;
    if (nc && it > 0) {  // the Jacobian K(V; U) and its diagonal at the new iterate
      e = nc_flags(c, U);
      if (e == cudaSuccess) e = launch_u_diag(E, c->f[VFGPU_FIELD_V], c->bcU_bits, JY, c->stream, U);
      if (e == cudaSuccess) e = dev_inv(JY, dinv, mixed ? c->p32[4] : nullptr, n3, c->stream);
      if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
    }
    if (o.pc == VFGPU_PC_MG) {
      int levels = 0;
      // FP64 Krylov vectors with a V-cycle in the solve's precision; the set-up is
      // kept across Newton steps unless NOCOMPRESSION re-formed the Jacobian
      rc = run_mgcg(c, mixed, F, Y, R, P, W, dinv, c->p32[4], it > 0 && !nc, o.ksp_rtol, o.ksp_atol,
                    o.ksp_dtol, o.ksp_maxit, &kits, &kreason, &levels);
      if (rc) return rc;
      S.ksp_its += kits;
      tmo = w.expired();
    } else if (!mixed) {
      CGVecs<double> v{Y, R, P, W, dinv, F, nullptr, n3, dot_buf(c, 1), u_dots_of(c, c->plan64, 8)};
      rc = run_cg<double>(c, 1, v, apply64, o.ksp_rtol, o.ksp_atol, o.ksp_dtol, o.ksp_maxit, w, &kits,
                          &kreason, &tmo);
      if (rc) return rc;
      S.ksp_its += kits;
    } else {
      // Iterative refinement: FP32 PCG corrections, FP64 residual F - J Y.
      e = cudaMemsetAsync(Y, 0, n3 * sizeof(double), c->stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(R, F, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
      if (e == cudaSuccess) e = dev_znorm2(F, dinv, n3, c->d_red, c->d_out, c->stream);
      if (e == cudaSuccess) e = fetch(c, 1);
      if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
      const double z0 = sqrt(c->h_out[0]), target = std::max(o.ksp_rtol * z0, o.ksp_atol);
      double zr = z0;
      kreason = CG_DIVERGED_ITS;
      for (int k = 0; k < o.max_refine && zr > target; k++) {
        float *x32 = c->p32[0], *r32 = c->p32[1], *pp32 = c->p32[2], *w32 = c->p32[3];
        float* b32 = reinterpret_cast<float*>(P);  // FP32 right-hand side staged in P
        e = dev_to_f32(R, b32, n3, c->stream);
        if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
        CGVecs<float> v{x32, r32, pp32, w32, c->p32[4], b32, nullptr, n3, dot_buf(c, 2), u_dots_of(c, c->plan32, 4)};
        const double in_rtol = std::max(o.inner_rtol, 0.5 * target / zr);
        int its32 = 0, r32reason = 0;
        rc = run_cg<float>(c, 2, v, apply32, in_rtol, 0.0, o.ksp_dtol, o.ksp_maxit, w, &its32,
                           &r32reason, &tmo);
        if (rc) return rc;
        S.ksp_its += its32;
        S.refine_its += 1;
        if (r32reason < 0 && r32reason != CG_DIVERGED_ITS && its32 == 0) break;
        e = dev_add_f32(Y, x32, n3, c->stream);
        if (e == cudaSuccess) e = u_apply64(c, Y, JY, nullptr);            // J Y (FP64)
        if (e == cudaSuccess) e = dev_axpby(R, F, -1.0, JY, n3, c->stream);  // R = F - J Y
        if (e == cudaSuccess) e = dev_znorm2(R, dinv, n3, c->d_red, c->d_out, c->stream);
        if (e == cudaSuccess) e = fetch(c, 1);
        if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
        zr = sqrt(c->h_out[0]);
        if (!(zr == zr)) {
          kreason = CG_DIVERGED_NAN;
          break;
        }
        if (tmo) break;
      }
      if (zr <= target) kreason = CG_CONVERGED_RTOL;
    }
    if (tmo) {
      reason = -100;  // wall-clock watchdog
      break;
    }
    if (kreason < 0 && kreason != CG_DIVERGED_ITS) {
      reason = -3;  // SNES_DIVERGED_LINEAR_SOLVE
      break;
    }
    double lambda = 1.0, ynorm = 0.;
    if (!nc) {
      // L2 line search.  F is affine in U, so ||F(U - l Y)||^2 is an exact quadratic in l
      // whose minimiser (what SNESLINESEARCHL2's secant step lands on) is
      // l* = (F . JY) / (JY . JY).
      e = u_apply64(c, Y, JY, nullptr);
      const double* pa[3] = {F, JY, Y};
      const double* pb[3] = {JY, JY, Y};
      if (e == cudaSuccess) e = dev_dots(pa, pb, 3, n3, c->d_red, c->d_out, c->stream);
      if (e == cudaSuccess) e = fetch(c, 3);
      if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
      if (c->h_out[1] > 0) {
        const double l = c->h_out[0] / c->h_out[1];
        if (l == l && l > 1e-12) lambda = l;
      }
      ynorm = lambda * sqrt(c->h_out[2]);
      e = dev_axpy(U, -lambda, Y, n3, c->stream);
      if (e == cudaSuccess) e = u_residual(c, U, f, JY, F);
    } else {
      // L2 line search on the piecewise-affine NOCOMPRESSION residual: one secant step
      // on the derivative of ||F(U - l Y)||^2 fitted through l = 0, 1/2, 1.
      double q[2];
      for (int sidx = 0; sidx < 2; sidx++) {
        e = cudaMemcpyAsync(W, U, n3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = dev_axpy(W, sidx == 0 ? -0.5 : -1.0, Y, n3, c->stream);
        if (e == cudaSuccess) e = nc_residual(W, R);
        q[sidx] = dot_host(c, R, R, n3, e);
        if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
      }
      const double q0 = fnorm * fnorm, qm = q[0], q1 = q[1];
      const double dE = 3. * q1 - 4. * qm + q0, dE_old = -3. * q0 + 4. * qm - q1;
      if (dE - dE_old != 0.) {
        const double lu = 1. - dE / (dE - dE_old);
        if (lu == lu && lu > 1e-12) lambda = lu;
      }
      ynorm = lambda * sqrt(dot_host(c, Y, Y, n3, e));
      if (e == cudaSuccess) e = dev_axpy(U, -lambda, Y, n3, c->stream);
      if (e == cudaSuccess) e = nc_residual(U, F);
    }
    const double* qa[2] = {F, U};
    const double* qb[2] = {F, U};
    if (e == cudaSuccess) e = dev_dots(qa, qb, 2, n3, c->d_red, c->d_out, c->stream);
    if (e == cudaSuccess) e = fetch(c, 2);
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_u");
    fnorm = sqrt(c->h_out[0]);
    const double xnorm = sqrt(c->h_out[1]);
    S.newton_its = it + 1;
    if (!(fnorm == fnorm)) reason = -4;                 // SNES_DIVERGED_FNORM_NAN
    else if (fnorm < o.snes_atol) reason = 2;           // SNES_CONVERGED_FNORM_ABS
    else if (fnorm <= ttol) reason = 3;                 // SNES_CONVERGED_FNORM_RELATIVE
    else if (ynorm < o.snes_stol * xnorm) reason = 4;   // SNES_CONVERGED_SNORM_RELATIVE
    if (w.expired() && !reason) reason = -100;
  }
  if (!reason) reason = -5;  // SNES_DIVERGED_MAX_IT
  if (int rc2 = check_cell_copies(c)) return rc2;
  S.reason = reason;
  S.fnorm = fnorm;
  S.seconds = w.seconds();
  if (st) *st = S;
  if (reason > 0) return VFGPU_OK;
  if (reason == -5 || reason == -100) return VFGPU_NOT_CONVERGED;
  return VFGPU_DIVERGED;
}

}  // extern "C"

namespace vfgpu {

// ---------------------------------------------------------------------------- V
static cudaError_t v_apply64(vfgpu_ctx* c, const double* x, double* y, const uint8_t* mask,
                             const int* skip, double* dot = nullptr) {
  VApplyArgs<double> A = v_args<double>(c, x, y, mask, c->vmap64, c->seam64, c->vplan64);
  A.skip = skip;
  A.dot = dot;
  return launch_v_apply<double>(A, c->vplan64, c->layers, c->stream);
}
static cudaError_t v_apply32(vfgpu_ctx* c, const float* x, float* y, const uint8_t* mask,
                             const int* skip, double* dot = nullptr) {
  VApplyArgs<float> A = v_args<float>(c, x, y, mask, c->vmap32, c->seam32, c->vplan32);
  A.skip = skip;
  A.dot = dot;
  return launch_v_apply<float>(A, c->vplan32, c->layers, c->stream);
}

// F_V (VF_VResidual, VFMech.c:2687-2879) at v.
static cudaError_t v_residual(vfgpu_ctx* c, const double* v, const double* b, double* tmp,
                              double* F) {
  cudaError_t e = v_apply64(c, v, tmp, nullptr, nullptr);
  if (e == cudaSuccess)
    e = dev_v_residual(tmp, b, v, c->f[VFGPU_FIELD_VIRREV], c->bcV_kind, c->vf.irrevtol,
                       c->vf.atnum == 2, F, c->N, c->stream);
  return e;
}

}  // namespace vfgpu

extern "C" {

int vfgpu_step_v(vfgpu_ctx* c, const vfgpu_solve_opts* o_, vfgpu_solve_stats* st) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_step_v: null ctx");
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "vfgpu_step_v: material not set");
  vfgpu_solve_opts o;
  if (o_) o = *o_; else vfgpu_default_solve_opts(&o);
  if (o.precision != VFGPU_FP64 && o.precision != VFGPU_MIXED)
    return fail(VFGPU_ERR_INVALID, "vfgpu_step_v: bad precision");
  vfgpu_solve_stats S{};
  cudaSetDevice(c->dev);
  int rc = solve_buffers(c);
  if (rc) return rc;
  Watch w;
  w.limit = o.time_limit;
  const int64_t N = c->N;
  const bool mixed = o.precision == VFGPU_MIXED, at2 = c->vf.atnum == 2;
  // N-sized work vectors carved from the 3N pools at 16-byte aligned offsets (the CG
  // kernels use 16-byte accesses)
  const int64_t Na = pool_stride(N);
  double *lb = c->p64[0], *ub = c->p64[0] + Na, *b = c->p64[0] + 2 * Na;
  double *dinv = c->p64[1], *F = c->p64[1] + Na, *Y = c->p64[1] + 2 * Na;
  double *Wt = c->p64[2], *Fw = c->p64[2] + Na, *tmp = c->p64[2] + 2 * Na;
  double *R = c->p64[3], *P = c->p64[3] + Na, *Wv = c->p64[3] + 2 * Na;
  double* Vy = c->p64[4];  // N: accumulated correction of the mixed solve
  float *dinv32 = c->p32[4], *x32 = c->p32[0], *r32 = c->p32[1], *pp32 = c->p32[2], *w32 = c->p32[3];
  float* b32 = c->p32[4] + Na;
  double* V = c->f[VFGPU_FIELD_V];
  uint8_t* mask = c->vmask;
  ElemArgs E = elem_args(c);
  c->v32_stale = c->ul_stale = true;  // V changes from here on, also on an error return
  cudaError_t e = dev_v_bounds(c->f[VFGPU_FIELD_VIRREV], c->vf.atnum == 1, lb, ub, V, N, c->stream);
  if (e == cudaSuccess)
    e = launch_v_coef(E, c->f[VFGPU_FIELD_U], c->f[VFGPU_FIELD_THETA], c->f[VFGPU_FIELD_THETAREF],
                      c->coef64, mixed ? c->coef32 : nullptr, c->stream);
  if (e == cudaSuccess) e = launch_v_rhs(E, c->f[VFGPU_FIELD_U], c->f[VFGPU_FIELD_PRESSURE], b, c->stream);
  if (e == cudaSuccess) e = launch_v_diag(E, c->coef64, tmp, c->stream);
  if (e == cudaSuccess) e = dev_inv(tmp, dinv, mixed ? dinv32 : nullptr, N, c->stream);
  if (e == cudaSuccess) e = v_residual(c, V, b, tmp, F);
  if (e == cudaSuccess) e = dev_vi_norm2(F, V, lb, ub, N, c->d_red, c->d_out, c->stream);
  if (e == cudaSuccess) e = fetch(c, 1);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
  double fnorm = sqrt(c->h_out[0]);
  S.fnorm0 = fnorm;
  const double ttol = o.snes_rtol * fnorm;
  int reason = 0;
  if (fnorm < o.snes_atol) reason = 2;
  auto apply64 = [&](const double* x, double* y, const int* skip, double* dot) {
    return v_apply64(c, x, y, mask, skip, dot);
  };
  auto apply32 = [&](const float* x, float* y, const int* skip, double* dot) {
    return v_apply32(c, x, y, mask, skip, dot);
  };
  for (int it = 0; !reason && it < o.snes_maxit; it++) {
    e = dev_v_mask(F, V, lb, ub, c->f[VFGPU_FIELD_VIRREV], c->bcV_kind, c->vf.irrevtol, at2, mask, N,
                   c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
    int kits = 0, kreason = 0;
    bool tmo = false;
    if (!mixed) {
      CGVecs<double> v{Y, R, P, Wv, dinv, F, mask, N, dot_buf(c, 3), dots_of(c, c->vplan64)};
      rc = run_cg<double>(c, 3, v, apply64, o.ksp_rtol, o.ksp_atol, o.ksp_dtol, o.ksp_maxit, w, &kits,
                          &kreason, &tmo);
      if (rc) return rc;
      S.ksp_its += kits;
    } else {
      e = cudaMemsetAsync(Vy, 0, N * sizeof(double), c->stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(R, F, N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
      if (e == cudaSuccess) e = dev_v_fix_step(R, F, mask, nullptr, N, c->stream);  // R = 0 on removed dofs
      if (e == cudaSuccess) e = dev_znorm2(R, dinv, N, c->d_red, c->d_out, c->stream);
      if (e == cudaSuccess) e = fetch(c, 1);
      if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
      const double z0 = sqrt(c->h_out[0]), target = std::max(o.ksp_rtol * z0, o.ksp_atol);
      double zr = z0;
      kreason = zr <= target ? CG_CONVERGED_ATOL : CG_DIVERGED_ITS;
      for (int k = 0; k < o.max_refine && zr > target; k++) {
        e = dev_to_f32(R, b32, N, c->stream);
        if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
        CGVecs<float> v{x32, r32, pp32, w32, dinv32, b32, mask, N, dot_buf(c, 4), dots_of(c, c->vplan32)};
        const double in_rtol = std::max(o.inner_rtol, 0.5 * target / zr);
        int its32 = 0, r32reason = 0;
        rc = run_cg<float>(c, 4, v, apply32, in_rtol, 0.0, o.ksp_dtol, o.ksp_maxit, w, &its32,
                           &r32reason, &tmo);
        if (rc) return rc;
        S.ksp_its += its32;
        S.refine_its += 1;
        e = dev_add_f32(Vy, x32, N, c->stream);
        if (e == cudaSuccess) e = v_apply64(c, Vy, tmp, mask, nullptr);
        if (e == cudaSuccess) e = dev_axpby(R, F, -1.0, tmp, N, c->stream);
        if (e == cudaSuccess) e = dev_v_fix_step(R, F, mask, nullptr, N, c->stream);
        if (e == cudaSuccess) e = dev_znorm2(R, dinv, N, c->d_red, c->d_out, c->stream);
        if (e == cudaSuccess) e = fetch(c, 1);
        if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
        zr = sqrt(c->h_out[0]);
        if (!(zr == zr)) {
          kreason = CG_DIVERGED_NAN;
          break;
        }
        if (tmo) break;
      }
      if (zr <= target) kreason = CG_CONVERGED_RTOL;
      e = cudaMemcpyAsync(Y, Vy, N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
      if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
    }
    if (tmo) {
      reason = -100;
      break;
    }
    if (kreason < 0 && kreason != CG_DIVERGED_ITS) {
      reason = -3;
      break;
    }
    e = dev_v_fix_step(Y, F, mask, c->bcV_kind, N, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
    // projected back-tracking line search (SNESLINESEARCHBT with alpha = 0): accept the
    // first lambda = 1, 1/2, ... that does not increase the inactive-set norm.
    double lambda = 1.0, gnorm = 0.0, ynorm2 = 0.0;
    for (int bt = 0; bt < 30; bt++) {
      e = dev_v_project(V, Y, lambda, lb, ub, Wt, N, c->d_red, c->d_out, c->stream);
      if (e == cudaSuccess) e = fetch(c, 1);
      ynorm2 = c->h_out[0];
      if (e == cudaSuccess) e = v_residual(c, Wt, b, tmp, Fw);
      if (e == cudaSuccess) e = dev_vi_norm2(Fw, Wt, lb, ub, N, c->d_red, c->d_out, c->stream);
      if (e == cudaSuccess) e = fetch(c, 1);
      if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
      gnorm = sqrt(c->h_out[0]);
      if (gnorm <= fnorm || lambda < 1e-12) break;
      lambda *= 0.5;
    }
    e = cudaMemcpyAsync(V, Wt, N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(F, Fw, N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    const double xnorm = sqrt(dot_host(c, V, V, N, e));
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_step_v");
    fnorm = gnorm;
    const double ynorm = sqrt(ynorm2);
    S.newton_its = it + 1;
    if (!(fnorm == fnorm)) reason = -4;
    else if (fnorm < o.snes_atol) reason = 2;
    else if (fnorm <= ttol) reason = 3;
    else if (ynorm < o.snes_stol * xnorm) reason = 4;
    if (w.expired() && !reason) reason = -100;
  }
  if (!reason) reason = -5;
  c->v32_stale = c->ul_stale = true;
  if (int rc2 = check_cell_copies(c)) return rc2;
  S.reason = reason;
  S.fnorm = fnorm;
  S.seconds = w.seconds();
  if (st) *st = S;
  if (reason > 0) return VFGPU_OK;
  if (reason == -5 || reason == -100) return VFGPU_NOT_CONVERGED;
  return VFGPU_DIVERGED;
}

// VFTimeStepPrepare (VFCommon.c:1132-1157): VIrrev := V, U and V take their
// Dirichlet values; the AT1 upper bound is VIrrev (applied inside vfgpu_step_v).
int vfgpu_time_step_prepare(vfgpu_ctx* c) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_time_step_prepare: null ctx");
  cudaSetDevice(c->dev);
  // the multigrid eigenvalue estimates restart from their seed at each time step, so a
  // time step's results do not depend on the problems a pooled ctx solved before
  c->mg_ev = false;
  c->v32_stale = c->ul_stale = true;
  cudaError_t e = cudaMemcpyAsync(c->f[VFGPU_FIELD_VIRREV], c->f[VFGPU_FIELD_V], c->N * sizeof(double),
                                  cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = dev_apply_bc(c->f[VFGPU_FIELD_U], c->bcU_kind, c->f[VFGPU_FIELD_BCU], 3 * c->N, c->stream);
  if (e == cudaSuccess) e = dev_apply_bc(c->f[VFGPU_FIELD_V], c->bcV_kind, nullptr, c->N, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_time_step_prepare");
  return VFGPU_OK;
}

// One alternate-minimisation iteration: VF_StepU then VF_StepV, and ||V - Vold||_inf
// (the loop body of VFFractureTimeStep, VFCommon.c:1183-1202).
int vfgpu_am_step(vfgpu_ctx* c, const vfgpu_solve_opts* o, double* errV, vfgpu_solve_stats* su,
                  vfgpu_solve_stats* sv) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_am_step: null ctx");
  cudaSetDevice(c->dev);
  int rc = solve_buffers(c);
  if (rc) return rc;
  double* vold = c->p64[8];
  cudaError_t e = cudaMemcpyAsync(vold, c->f[VFGPU_FIELD_V], c->N * sizeof(double),
                                  cudaMemcpyDeviceToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_am_step");
  int ru = vfgpu_step_u(c, o, su);
  if (ru < 0) return ru;
  int rv = vfgpu_step_v(c, o, sv);
  if (rv < 0) return rv;
  e = dev_absmax_diff(c->f[VFGPU_FIELD_V], vold, c->N, c->d_red, c->d_out, c->stream);
  if (e == cudaSuccess) e = fetch(c, 1);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_am_step");
  if (errV) *errV = c->h_out[0];
  return std::max(ru, rv);
}

static int energies(vfgpu_ctx* c, double* cellcov) {
  if (!c) return fail(VFGPU_ERR_INVALID, "null ctx");
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "material not set");
  cudaSetDevice(c->dev);
  int rc = solve_buffers(c);
  if (rc) return rc;
  double* cc = cellcov;
  const bool stage = cellcov && !is_device_ptr(cellcov);
  if (stage) cc = c->p64[8];
  ElemArgs E = elem_args(c);
  cudaError_t e = launch_energies(E, c->f[VFGPU_FIELD_U], c->f[VFGPU_FIELD_V], c->f[VFGPU_FIELD_THETA],
                                  c->f[VFGPU_FIELD_THETAREF], c->f[VFGPU_FIELD_PRESSURE],
                                  c->d_red + RED_BLOCKS * 4, c->d_out, cc, c->stream);
  // d_out[4] = in-situ work (partials in the CG part of d_red, idle outside solves)
  if (e == cudaSuccess && c->has_insitu)
    e = launch_insitu_work(insitu_args(c), c->f[VFGPU_FIELD_U], c->d_red, c->d_out + 4, c->stream);
  else if (e == cudaSuccess)
    e = cudaMemsetAsync(c->d_out + 4, 0, sizeof(double), c->stream);
  if (e == cudaSuccess && stage)
    e = cudaMemcpyAsync(cellcov, cc, c->NC * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = fetch(c, 5);
  if (e != cudaSuccess) return cuda_fail(e, "energies");
  return VFGPU_OK;
}

int vfgpu_u_energy(vfgpu_ctx* c, double* elastic, double* insitu, double* pressurework) {
  int rc = energies(c, nullptr);
  if (rc) return rc;
  if (elastic) *elastic = c->h_out[0];
  if (insitu) *insitu = c->h_out[4];
  if (pressurework) *pressurework = c->h_out[1];
  return VFGPU_OK;
}

int vfgpu_v_energy(vfgpu_ctx* c, double* surface) {
  int rc = energies(c, nullptr);
  if (rc) return rc;
  if (surface) *surface = c->h_out[2];
  return VFGPU_OK;
}

int vfgpu_crack_opening(vfgpu_ctx* c, double* cov, double* cellcov) {
  int rc = energies(c, cellcov);
  if (rc) return rc;
  if (cov) *cov = c->h_out[3];
  return VFGPU_OK;
}

int vfgpu_memory_estimate(const vfgpu_grid* g, long long* bytes) {
  if (!g || !bytes) return fail(VFGPU_ERR_INVALID, "vfgpu_memory_estimate: null argument");
  if (g->nx < 2 || g->ny < 2 || g->nz < 2)
    return fail(VFGPU_ERR_INVALID, "vfgpu_memory_estimate: bad grid");
  const long long N = (long long)g->nx * g->ny * g->nz;
  const long long NC = (long long)(g->nx - 1) * (g->ny - 1) * (g->nz - 1);
  const TilePlan p64 = u_plan(g->nx, g->ny, g->nz, 8, 148), p32 = u_plan(g->nx, g->ny, g->nz, 4, 148);
  const TilePlan q64 = v_plan(g->nx, g->ny, g->nz, 8, 148), q32 = v_plan(g->nx, g->ny, g->nz, 4, 148);
  long long b = 0;
  b += (2 * 3 * N + 5 * N) * 8;                          // fields U, BCU, V, VIrrev, theta, thetaRef, p
  b += N * 4 + (g->nz - 1) + 3 * N + 3 * N;              // V32, layers, BC kinds and bits
  b += (long long)(unit_lists_bytes(p64, g->nz) + unit_lists_bytes(p32, g->nz));  // U unit lists
  b += (long long)std::max(p64.seamX + p64.seamY, q64.seamX + q64.seamY) * 8 +
       (long long)std::max(p32.seamX + p32.seamY, q32.seamX + q32.seamY) * 4;
  b += 3 * 3 * N * 8 + 2 * 3 * N * 4;                    // staging vectors
  b += vfgpu_ctx::NP64 * (3 * N + kPoolSlack) * 8 + vfgpu_ctx::NP32 * (3 * N + kPoolSlack) * 4;
  b += vcoef_size(g->nx - 1, g->ny - 1, g->nz - 1) * 12 + N;  // V coefficient (FP64 + FP32), mask
  b += (RED_BLOCKS + energy_blocks()) * 4 * 8 + 4096;    // reductions, scalars
  *bytes = b;
  return VFGPU_OK;
}

int vfgpu_u_residual(vfgpu_ctx* c, double* F) {
  if (!c || !F) return fail(VFGPU_ERR_INVALID, "vfgpu_u_residual: null argument");
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "vfgpu_u_residual: material not set");
  cudaSetDevice(c->dev);
  int rc = solve_buffers(c);
  if (rc) return rc;
  ElemArgs E = elem_args(c);
  double *f = c->p64[0], *tmp = c->p64[1], *Fd = c->p64[2];
  cudaError_t e = u_lists_refresh(c);
  if (e == cudaSuccess) e = nc_flags(c, c->f[VFGPU_FIELD_U]);
  if (e == cudaSuccess) e = u_load(c, E, f, c->f[VFGPU_FIELD_U]);
  if (e == cudaSuccess) e = u_residual(c, c->f[VFGPU_FIELD_U], f, tmp, Fd);
  if (e == cudaSuccess) e = copy_out(c, F, Fd, 3 * c->N);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_residual");
  return VFGPU_OK;
}

int vfgpu_v_residual(vfgpu_ctx* c, double* F) {
  if (!c || !F) return fail(VFGPU_ERR_INVALID, "vfgpu_v_residual: null argument");
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "vfgpu_v_residual: material not set");
  cudaSetDevice(c->dev);
  int rc = solve_buffers(c);
  if (rc) return rc;
  ElemArgs E = elem_args(c);
  const int64_t N = c->N;
  const int64_t Na = pool_stride(N);
  double *b = c->p64[0], *tmp = c->p64[0] + Na, *Fd = c->p64[0] + 2 * Na;
  cudaError_t e = launch_v_coef(E, c->f[VFGPU_FIELD_U], c->f[VFGPU_FIELD_THETA],
                                c->f[VFGPU_FIELD_THETAREF], c->coef64, nullptr, c->stream);
  if (e == cudaSuccess) e = launch_v_rhs(E, c->f[VFGPU_FIELD_U], c->f[VFGPU_FIELD_PRESSURE], b, c->stream);
  if (e == cudaSuccess) e = v_residual(c, c->f[VFGPU_FIELD_V], b, tmp, Fd);
  if (e == cudaSuccess) e = copy_out(c, F, Fd, N);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_v_residual");
  return check_cell_copies(c);
}

}  // extern "C"
