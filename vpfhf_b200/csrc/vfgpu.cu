// vfgpu.cu -- C ABI: context life cycle, material / BC / field set-up and the
// operator entry points.  See include/vfgpu.h for the contract.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include <algorithm>

#include "abi_util.h"
#include "ctx.h"
#include "vec.h"

using namespace vfgpu;

namespace vfgpu {

static thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation)
    return fail(VFGPU_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
  return fail(VFGPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int64_t field_len(const vfgpu_ctx* c, int field) {
  return (field == VFGPU_FIELD_U || field == VFGPU_FIELD_BCU) ? 3 * c->N : c->N;
}

// Copies n doubles from src (host or device) into device dst on the ctx stream.
cudaError_t copy_in(vfgpu_ctx* c, double* dst, const double* src, int64_t n) {
  return cudaMemcpyAsync(dst, src, n * sizeof(double),
                         is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                         c->stream);
}
cudaError_t copy_out(vfgpu_ctx* c, double* dst, const double* src, int64_t n) {
  return cudaMemcpyAsync(dst, src, n * sizeof(double),
                         is_device_ptr(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                         c->stream);
}

// Per-dof BC kind with the precedence of VecApplyDirichletBC /
// ResidualApplyDirichletBC (VFCartFE.c:493-998): faces X0,X1,Y0,Y1,Z0,Z1 in that
// order (a later face wins on shared edges), then the vertices in the order the
// reference visits them.
static void build_bc_kind(int nx, int ny, int nz, int dof, const vfgpu_bc* bc,
                          std::vector<uint8_t>& kind) {
  const int64_t N = (int64_t)nx * ny * nz;
  kind.assign(N * dof, 0);
  auto set = [&](int i, int j, int k, int c, int t) {
    kind[(((int64_t)k * ny + j) * nx + i) * dof + c] = (uint8_t)t;
  };
  for (int c = 0; c < dof; c++) {
    for (int fc = 0; fc < 6; fc++) {
      const int t = bc[c].face[fc];
      if (t == VFGPU_BC_NONE) continue;
      if (fc < 2) {
        const int i = fc == 0 ? 0 : nx - 1;
        for (int k = 0; k < nz; k++)
          for (int j = 0; j < ny; j++) set(i, j, k, c, t);
      } else if (fc < 4) {
        const int j = fc == 2 ? 0 : ny - 1;
        for (int k = 0; k < nz; k++)
          for (int i = 0; i < nx; i++) set(i, j, k, c, t);
      } else {
        const int k = fc == 4 ? 0 : nz - 1;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) set(i, j, k, c, t);
      }
    }
    static const int order[8] = {0, 4, 2, 6, 1, 5, 3, 7};
    for (int o = 0; o < 8; o++) {
      const int vtx = order[o], t = bc[c].vertex[vtx];
      if (t == VFGPU_BC_NONE) continue;
      set((vtx & 1) ? nx - 1 : 0, (vtx & 2) ? ny - 1 : 0, (vtx & 4) ? nz - 1 : 0, c, t);
    }
  }
}

int ensure_v32(vfgpu_ctx* c) {
  if (!c->v32_stale) return VFGPU_OK;
  cudaError_t e = convert_f64_f32(c->f[VFGPU_FIELD_V], c->V32, c->N, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "V to FP32");
  c->v32_stale = false;
  return VFGPU_OK;
}

// Rewrites the device parameter block from the host-side material and vfprop.
int upload_params(vfgpu_ctx* c) {
  DevParams P{};
  P.L = c->layers;
  P.eta = c->vf.eta;
  const double atcv = c->vf.atnum == 1 ? 2. / 3. : .5;  // VFCommon.c:482-492
  for (int l = 0; l < VF_MAXLAYER; l++) P.aeps[l] = c->layers.Gc[l] / atcv * .5 * c->vf.epsilon;
  cudaError_t e = cudaMemcpyAsync(c->d_params, &P, sizeof P, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "parameter upload");
  return VFGPU_OK;
}

template <typename T>
UApplyArgs<T> u_args(vfgpu_ctx* c, const T* x, const T* v, T* y, T* seam, const TilePlan& p) {
  UApplyArgs<T> A{};
  A.x = x;
  A.v = v;
  A.y = y;
  A.bc = c->bcU_bits;
  A.elayer = c->d_elayer;
  A.cellE = c->d_cellE;
  A.seamX = seam;
  A.seamY = seam + p.seamX;
  A.nx = c->nx;
  A.ny = c->ny;
  A.nz = c->nz;
  A.ihx = T(1.0 / c->hx);
  A.ihy = T(1.0 / c->hy);
  A.ihz = T(1.0 / c->hz);
  A.vol = T(c->hx * c->hy * c->hz);
  A.eta = T(c->vf.eta);
  A.P = c->d_params;
  A.cflag = c->unilateral ? c->d_cflag : nullptr;
  use_unit_lists(A, u_lists_on(c, (int)sizeof(T)) ? (sizeof(T) == 8 ? c->ul64 : c->ul32) : UnitLists{});
  A.plane_err = c->d_cerr;
  return A;
}
// The split mode and the grid call for the lists in this precision (NOCOMPRESSION aside).
static bool u_lists_wanted(const vfgpu_ctx* c, int prec_bytes) {
  const TilePlan& p = prec_bytes == 8 ? c->plan64 : c->plan32;
  if (!(prec_bytes == 8 ? c->ul64.cls : c->ul32.cls)) return false;
  if (c->u_split == VFGPU_U_SPLIT_ON) return true;
  return c->u_split == VFGPU_U_SPLIT_AUTO && unit_lists_pay(p, c->nz, prec_bytes);
}

cudaError_t u_lists_refresh(vfgpu_ctx* c) {
  if (!c->ul_stale) return cudaSuccess;
  const double* v = c->f[VFGPU_FIELD_V];
  cudaError_t e = cudaSuccess;
  if (u_lists_wanted(c, 8)) e = build_unit_lists(v, c->nx, c->ny, c->nz, c->plan64, c->ul64, c->stream);
  if (e == cudaSuccess && u_lists_wanted(c, 4))
    e = build_unit_lists(v, c->nx, c->ny, c->nz, c->plan32, c->ul32, c->stream);
  if (e == cudaSuccess) c->ul_stale = false;
  return e;
}

bool u_lists_on(const vfgpu_ctx* c, int prec_bytes) {
  return !c->unilateral && u_lists_wanted(c, prec_bytes);
}

template UApplyArgs<double> u_args<double>(vfgpu_ctx*, const double*, const double*, double*,
                                           double*, const TilePlan&);
template UApplyArgs<float> u_args<float>(vfgpu_ctx*, const float*, const float*, float*, float*,
                                         const TilePlan&);

}  // namespace vfgpu

// ---------------------------------------------------------------------------
extern "C" {

const char* vfgpu_last_error(void) { return g_err.c_str(); }

int vfgpu_destroy(vfgpu_ctx* c) {
  if (!c) return VFGPU_OK;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& g : c->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  c->graphs.clear();
  free_solver(c);
  free_mg(c);
  for (auto& p : c->f) cudaFree(p);
  if (c->s_in) cudaStreamSynchronize(c->s_in);
  if (c->s_out) cudaStreamSynchronize(c->s_out);
  for (int s = 0; s < vfgpu_ctx::kPipeSlabs; s++)
    for (cudaEvent_t ev : {c->ev_in[s], c->ev_y[s], c->ev_out[s]})
      if (ev) cudaEventDestroy(ev);
  if (c->ev_start) cudaEventDestroy(c->ev_start);
  if (c->s_in) cudaStreamDestroy(c->s_in);
  if (c->s_out) cudaStreamDestroy(c->s_out);
  cudaFree(c->t64c);
  void* bufs[] = {c->d_tcB, c->d_tcerr, c->d_widthc, c->d_pmult, c->d_width, c->d_wpart, c->d_wstall, c->d_cflag, c->d_params, c->d_dot, c->d_elayer, c->d_ul, c->d_cerr, c->d_cellE, c->bcU_kind, c->bcU_bits, c->bcV_kind, c->bcV_bits,
                  c->V32, c->seam64, c->seam32, c->t64a, c->t64b, c->t32a, c->t32b};
  for (void* p : bufs) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return VFGPU_OK;
}

int vfgpu_create(const vfgpu_grid* g, vfgpu_ctx** out) {
  if (!g || !out) return fail(VFGPU_ERR_INVALID, "vfgpu_create: null argument");
  *out = nullptr;
  if (g->nx < 2 || g->ny < 2 || g->nz < 2)
    return fail(VFGPU_ERR_INVALID, "vfgpu_create: need at least 2 nodes per axis, got %d %d %d",
                g->nx, g->ny, g->nz);
  if (!(g->lx > 0) || !(g->ly > 0) || !(g->lz > 0))
    return fail(VFGPU_ERR_INVALID, "vfgpu_create: box lengths must be positive");
  if ((int64_t)g->nx * g->ny * g->nz * 3 >= (int64_t)1 << 31)
    return fail(VFGPU_ERR_INVALID, "vfgpu_create: grid too large for int32 dof indexing");
  vfgpu_ctx* c = new vfgpu_ctx();
  cudaError_t e = cudaGetDevice(&c->dev);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaGetDevice");
  }
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev);
  c->nx = g->nx;
  c->ny = g->ny;
  c->nz = g->nz;
  c->lx = g->lx;
  c->ly = g->ly;
  c->lz = g->lz;
  c->hx = g->lx / (g->nx - 1.);
  c->hy = g->ly / (g->ny - 1.);
  c->hz = g->lz / (g->nz - 1.);
  c->N = (int64_t)g->nx * g->ny * g->nz;
  c->NC = (int64_t)(g->nx - 1) * (g->ny - 1) * (g->nz - 1);
  c->plan64 = u_plan(c->nx, c->ny, c->nz, 8, c->nsm);
  c->plan32 = u_plan(c->nx, c->ny, c->nz, 4, c->nsm);
  c->vplan64 = v_plan(c->nx, c->ny, c->nz, 8, c->nsm);
  c->vplan32 = v_plan(c->nx, c->ny, c->nz, 4, c->nsm);
#define ALLOC(ptr, bytes)                                  \
  do {                                                     \
    e = cudaMalloc((void**)&(ptr), (size_t)(bytes));       \
    if (e != cudaSuccess) {                                \
      vfgpu_destroy(c);                                    \
      return cuda_fail(e, "vfgpu_create: cudaMalloc");     \
    }                                                      \
  } while (0)
  e = apply_kernel_attributes();
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "vfgpu_create: kernel attributes");
  }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    vfgpu_destroy(c);
    return cuda_fail(e, "cudaStreamCreate");
  }
  for (int fi = 0; fi < 7; fi++) ALLOC(c->f[fi], field_len(c, fi) * sizeof(double));
  ALLOC(c->V32, c->N * sizeof(float));
  ALLOC(c->d_elayer, std::max(1, c->nz - 1));
  {
    const size_t b64 = unit_lists_bytes(c->plan64, c->nz), b32 = unit_lists_bytes(c->plan32, c->nz);
    if (b64 + b32 > 0) {
      ALLOC(c->d_ul, b64 + b32);
      c->ul64 = unit_lists_carve(b64 ? c->d_ul : nullptr, c->plan64, c->nz);
      c->ul32 = unit_lists_carve(b32 ? static_cast<char*>(c->d_ul) + b64 : nullptr, c->plan32, c->nz);
    }
  }
  ALLOC(c->d_params, sizeof(DevParams));
  ALLOC(c->d_cerr, sizeof(unsigned));
  {
    int nd = 1;
    for (const TilePlan* p : {&c->plan64, &c->plan32, &c->vplan64, &c->vplan32})
      nd = std::max(nd, tile_dot_count(*p, c->nx, c->ny, c->nz) + p->ncta0);  // U: split launch
    ALLOC(c->d_dot, (size_t)nd * sizeof(double));
  }
  ALLOC(c->bcU_kind, 3 * c->N);
  ALLOC(c->bcU_bits, c->N);
  ALLOC(c->bcV_kind, c->N);
  ALLOC(c->bcV_bits, c->N);
  // one seam buffer per precision serves the U and the V operator: the larger of the two
  // (the U operator's unless a build gives it taller tiles than the V operator's)
  ALLOC(c->seam64, std::max({(size_t)1, c->plan64.seamX + c->plan64.seamY,
                             c->vplan64.seamX + c->vplan64.seamY}) * sizeof(double));
  ALLOC(c->seam32, std::max({(size_t)1, c->plan32.seamX + c->plan32.seamY,
                             c->vplan32.seamX + c->vplan32.seamY}) * sizeof(float));
  ALLOC(c->t64a, 3 * c->N * sizeof(double));
  ALLOC(c->t64b, 3 * c->N * sizeof(double));
  ALLOC(c->t32a, 3 * c->N * sizeof(float));
  ALLOC(c->t32b, 3 * c->N * sizeof(float));
#undef ALLOC
  cudaMemsetAsync(c->d_elayer, 0, std::max(1, c->nz - 1), c->stream);
  cudaMemsetAsync(c->d_cerr, 0, sizeof(unsigned), c->stream);
  cudaMemsetAsync(c->bcU_kind, 0, 3 * c->N, c->stream);
  cudaMemsetAsync(c->bcU_bits, 0, c->N, c->stream);
  cudaMemsetAsync(c->bcV_kind, 0, c->N, c->stream);
  cudaMemsetAsync(c->bcV_bits, 0, c->N, c->stream);
  // VFFieldsInitialize defaults: U = BCU = 0, V = VIrrev = 1, theta = thetaRef = p = 0.
  for (int fi = 0; fi < 7; fi++) {
    const double val = (fi == VFGPU_FIELD_V || fi == VFGPU_FIELD_VIRREV) ? 1.0 : 0.0;
    e = fill_f64(c->f[fi], val, field_len(c, fi), c->stream);
    if (e != cudaSuccess) {
      vfgpu_destroy(c);
      return cuda_fail(e, "vfgpu_create: init fields");
    }
  }
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    vfgpu_destroy(c);
    return cuda_fail(e, "vfgpu_create");
  }
  if (upload_params(c) != VFGPU_OK) {
    vfgpu_destroy(c);
    return VFGPU_ERR_CUDA;
  }
  *out = c;
  return VFGPU_OK;
}

int vfgpu_set_matprop(vfgpu_ctx* c, int nlayer, const vfgpu_matprop* mp, const int* layer) {
  if (!c || !mp) return fail(VFGPU_ERR_INVALID, "vfgpu_set_matprop: null argument");
  if (nlayer < 1 || nlayer > VF_MAXLAYER)
    return fail(VFGPU_ERR_INVALID, "vfgpu_set_matprop: nlayer must be in [1,%d]", VF_MAXLAYER);
  cudaSetDevice(c->dev);
  c->mg_ev = false;  // a new material starts the multigrid eigenvalue estimates afresh
  c->mg_layers = false;  // ... and may move the element layers
  LayerTable L{};
  for (int l = 0; l < nlayer; l++) {
    const double E = mp[l].E, nu = mp[l].nu;
    if (!(E > 0) || !(nu > -1 && nu < 0.5))
      return fail(VFGPU_ERR_INVALID, "vfgpu_set_matprop: layer %d needs E > 0, -1 < nu < 0.5", l);
    // VFMatPropGet (VFCommon.c:583-586)
    L.lambda[l] = E * nu / (1. + nu) / (1. - 2. * nu);
    L.mu[l] = E / (1. + nu) * .5;
    L.lamfac[l] = nu / (1. + nu) / (1. - 2. * nu);
    L.mufac[l] = 1. / (1. + nu) * .5;
    L.alpha[l] = mp[l].alpha;
    L.beta[l] = mp[l].beta;
    L.Gc[l] = mp[l].Gc;
  }
  std::vector<uint8_t> el(std::max(1, c->nz - 1), 0);
  if (layer)
    for (int k = 0; k < c->nz - 1; k++) {
      if (layer[k] < 0 || layer[k] >= nlayer)
        return fail(VFGPU_ERR_INVALID, "vfgpu_set_matprop: layer[%d] = %d out of range", k,
                    layer[k]);
      el[k] = (uint8_t)layer[k];
    }
  cudaError_t e = cudaMemcpyAsync(c->d_elayer, el.data(), el.size(), cudaMemcpyHostToDevice,
                                  c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_set_matprop");
  c->layers = L;
  c->nlayer = nlayer;
  c->have_mat = true;
  return upload_params(c);
}

int vfgpu_set_cell_modulus(vfgpu_ctx* c, const double* cellE) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_set_cell_modulus: null ctx");
  cudaSetDevice(c->dev);
  // The cell-modulus pointer is captured by CG graphs: they are re-captured whenever it
  // appears, disappears or moves.
  if (!cellE) {
    if (c->d_cellE) c->gen++;
    cudaFree(c->d_cellE);
    c->d_cellE = nullptr;
    return VFGPU_OK;
  }
  cudaError_t e = cudaSuccess;
  if (!c->d_cellE) {
    c->gen++;
    e = cudaMalloc((void**)&c->d_cellE, c->NC * sizeof(float));
  }
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_set_cell_modulus");
  // staged through t64a (>= 3N >= NC doubles)
  e = copy_in(c, c->t64a, cellE, c->NC);
  if (e == cudaSuccess) e = convert_f64_f32(c->t64a, c->d_cellE, c->NC, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_set_cell_modulus");
  return VFGPU_OK;
}

int vfgpu_set_vfprop(vfgpu_ctx* c, const vfgpu_vfprop* vf) {
  if (!c || !vf) return fail(VFGPU_ERR_INVALID, "vfgpu_set_vfprop: null argument");
  if (vf->atnum != 1 && vf->atnum != 2)  // VFCommon.c:489-491
    return fail(VFGPU_ERR_INVALID, "vfgpu_set_vfprop: atnum should be 1 or 2, got %d", vf->atnum);
  if (!(vf->epsilon > 0) || !(vf->eta >= 0))
    return fail(VFGPU_ERR_INVALID, "vfgpu_set_vfprop: need epsilon > 0 and eta >= 0");
  c->vf = *vf;
  return upload_params(c);
}

int vfgpu_set_unilateral(vfgpu_ctx* c, int type) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_set_unilateral: null ctx");
  if (type != VFGPU_UNILATERAL_NONE && type != VFGPU_UNILATERAL_NOCOMPRESSION)
    return fail(VFGPU_ERR_INVALID, "vfgpu_set_unilateral: unknown type %d", type);
  cudaSetDevice(c->dev);
  if (type == VFGPU_UNILATERAL_NOCOMPRESSION && !c->d_cflag) {
    cudaError_t e = cudaMalloc((void**)&c->d_cflag, std::max<int64_t>(1, c->NC) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_cflag, 0, std::max<int64_t>(1, c->NC) * sizeof(uint32_t), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      cudaFree(c->d_cflag);
      c->d_cflag = nullptr;
      return cuda_fail(e, "vfgpu_set_unilateral");
    }
  }
  if (type != c->unilateral) c->gen++;  // captured CG graphs launch the other operator kernel
  c->unilateral = type;
  return VFGPU_OK;
}

int vfgpu_set_u_split(vfgpu_ctx* c, int mode) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_set_u_split: null ctx");
  if (mode != VFGPU_U_SPLIT_AUTO && mode != VFGPU_U_SPLIT_OFF && mode != VFGPU_U_SPLIT_ON)
    return fail(VFGPU_ERR_INVALID, "vfgpu_set_u_split: bad mode %d", mode);
  if (mode != c->u_split) {
    c->u_split = mode;
    c->ul_stale = true;  // lists of a precision that was off were not kept up to date
    c->gen++;            // captured CG graphs launch the other kernels
  }
  return VFGPU_OK;
}

int vfgpu_set_insitu(vfgpu_ctx* c, const double* smin, const double* smax) {
  if (!c) return fail(VFGPU_ERR_INVALID, "vfgpu_set_insitu: null ctx");
  c->has_insitu = smin != nullptr;
  for (int i = 0; i < 6; i++) {
    c->insitu_min[i] = smin ? smin[i] : 0.;
    c->insitu_max[i] = smin ? (smax ? smax[i] : smin[i]) : 0.;
    if (!(c->insitu_min[i] == c->insitu_min[i]) || !(c->insitu_max[i] == c->insitu_max[i]))
      return fail(VFGPU_ERR_INVALID, "vfgpu_set_insitu: NaN stress component %d", i);
  }
  return VFGPU_OK;
}

int vfgpu_set_bc(vfgpu_ctx* c, const vfgpu_bc bcU[3], const vfgpu_bc* bcV) {
  if (!c || !bcU || !bcV) return fail(VFGPU_ERR_INVALID, "vfgpu_set_bc: null argument");
  for (int k = 0; k < 4; k++) {
    const vfgpu_bc& b = k < 3 ? bcU[k] : *bcV;
    for (int f = 0; f < 6; f++)
      if (b.face[f] < 0 || b.face[f] > 3) return fail(VFGPU_ERR_INVALID, "vfgpu_set_bc: bad face type");
    for (int v = 0; v < 8; v++)
      if (b.vertex[v] < 0 || b.vertex[v] > 3)
        return fail(VFGPU_ERR_INVALID, "vfgpu_set_bc: bad vertex type");
  }
  cudaSetDevice(c->dev);
  std::vector<uint8_t> ku, kv, bu(c->N, 0), bv(c->N, 0);
  build_bc_kind(c->nx, c->ny, c->nz, 3, bcU, ku);
  build_bc_kind(c->nx, c->ny, c->nz, 1, bcV, kv);
  for (int64_t n = 0; n < c->N; n++) {
    for (int k = 0; k < 3; k++)
      if (ku[3 * n + k]) bu[n] |= (uint8_t)(1u << k);
    if (kv[n]) bv[n] = 1;
  }
  cudaError_t e = cudaMemcpyAsync(c->bcU_kind, ku.data(), ku.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->bcU_bits, bu.data(), bu.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->bcV_kind, kv.data(), kv.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->bcV_bits, bv.data(), bv.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_set_bc");
  for (int k = 0; k < 3; k++) c->bcU[k] = bcU[k];
  c->bcV = *bcV;
  return VFGPU_OK;
}

int vfgpu_set_field(vfgpu_ctx* c, int field, const double* data) {
  if (!c || !data) return fail(VFGPU_ERR_INVALID, "vfgpu_set_field: null argument");
  if (field < 0 || field > 6) return fail(VFGPU_ERR_INVALID, "vfgpu_set_field: bad field %d", field);
  cudaSetDevice(c->dev);
  if (field == VFGPU_FIELD_V) c->v32_stale = c->ul_stale = true;
  cudaError_t e = copy_in(c, c->f[field], data, field_len(c, field));
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_set_field");
  return VFGPU_OK;
}

int vfgpu_get_field(vfgpu_ctx* c, int field, double* data) {
  if (!c || !data) return fail(VFGPU_ERR_INVALID, "vfgpu_get_field: null argument");
  if (field < 0 || field > 6) return fail(VFGPU_ERR_INVALID, "vfgpu_get_field: bad field %d", field);
  cudaSetDevice(c->dev);
  cudaError_t e = copy_out(c, data, c->f[field], field_len(c, field));
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_get_field");
  return VFGPU_OK;
}

namespace {

// Streams, events and the second staging vector of the host-buffer pipeline.
cudaError_t pipe_resources(vfgpu_ctx* c) {
  if (c->t64c) return cudaSuccess;
  cudaError_t e = cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming);
  for (int s = 0; s < vfgpu_ctx::kPipeSlabs && e == cudaSuccess; s++)
    for (cudaEvent_t* ev : {&c->ev_in[s], &c->ev_y[s], &c->ev_out[s]})
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->t64c, 3 * c->N * sizeof(double));
  return e;
}

// y = K x with x and y in host memory (FP64), as a pipeline over z-slabs of node planes:
// slab s's planes go up on s_in, the slab with one halo plane on each side is applied
// as a sub-grid on the ctx stream (same xy tiles and per-node sum order as the whole-grid
// apply, so its interior planes carry the same bits; the halo planes' values are
// discarded), and its interior planes come back on s_out while later slabs are still
// going up, so that both copy directions and the compute overlap.  Slabs alternate
// between two output staging vectors, because a slab's apply also writes its halo
// planes, which belong to its neighbours.
cudaError_t u_apply_host_pipelined(vfgpu_ctx* c, const double* x, double* y) {
  cudaError_t e = pipe_resources(c);
  if (e != cudaSuccess) return e;
  // slabs of at least 4 planes, at most kPipeSlabs of them
  const int nz = c->nz, S = std::max(2, std::min(vfgpu_ctx::kPipeSlabs, nz / 4));
  const int64_t plane = (int64_t)c->nx * c->ny, cplane = (int64_t)(c->nx - 1) * (c->ny - 1);
  const int P = (nz + S - 1) / S;
  if (c->unilateral) e = nc_flags(c, c->f[VFGPU_FIELD_U]);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_start, c->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_in, c->ev_start, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_out, c->ev_start, 0);
  int up = 0;  // planes [0, up) are on their way up
  for (int s = 0; s < S && e == cudaSuccess; s++) {
    const int a = s * P, b = std::min(nz, (s + 1) * P);
    if (a >= b) break;
    const int lo = std::max(a - 1, 0), hi = std::min(b + 1, nz);
    if (hi > up) {
      e = cudaMemcpyAsync(c->t64a + 3 * up * plane, x + 3 * up * plane,
                          3 * (hi - up) * plane * sizeof(double), cudaMemcpyHostToDevice, c->s_in);
      up = hi;
    }
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_in[s], c->s_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_in[s], 0);
    double* buf = (s & 1) ? c->t64c : c->t64b;
    if (e == cudaSuccess) {
      const int nzs = hi - lo;
      const TilePlan p = u_plan(c->nx, c->ny, nzs, 8, c->nsm);
      UApplyArgs<double> A = u_args<double>(c, c->t64a + 3 * lo * plane, c->f[VFGPU_FIELD_V] + lo * plane,
                                            buf + 3 * lo * plane, c->seam64, p);
      A.nz = nzs;
      A.bc = c->bcU_bits + lo * plane;
      A.elayer = c->d_elayer + lo;
      use_unit_lists(A, UnitLists{});  // a sub-grid: the whole grid's lists do not apply
      if (A.cellE) A.cellE += lo * cplane;
      if (A.cflag) A.cflag += lo * cplane;
      e = launch_u_apply<double>(A, p, c->layers, c->stream);
    }
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_y[s], c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->s_out, c->ev_y[s], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(y + 3 * a * plane, buf + 3 * a * plane, 3 * (b - a) * plane * sizeof(double),
                          cudaMemcpyDeviceToHost, c->s_out);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_out[s], c->s_out);
    // the slab two ahead reuses this buffer's halo planes only: no wait is needed for
    // correctness; the ctx stream waits for the last copy out before returning
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->s_out);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e;
}

}  // namespace

int vfgpu_u_apply(vfgpu_ctx* c, int precision, const double* x, double* y) {
  if (!c || !x || !y) return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply: null argument");
  if (precision != VFGPU_FP64 && precision != VFGPU_MIXED)
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply: bad precision %d", precision);
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "vfgpu_u_apply: material not set");
  cudaSetDevice(c->dev);
  const int64_t n3 = 3 * c->N;
  const bool xdev = is_device_ptr(x), ydev = is_device_ptr(y);
  cudaError_t e = u_lists_refresh(c);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply");
  if (precision == VFGPU_FP64 && !xdev && !ydev && c->nz >= 8) {
    e = u_apply_host_pipelined(c, x, y);
    if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply");
    return VFGPU_OK;
  }
  const double* xd = x;
  if (!xdev) {
    e = copy_in(c, c->t64a, x, n3);
    xd = c->t64a;
  }
  double* yd = ydev ? y : c->t64b;
  if (e == cudaSuccess && c->unilateral) e = nc_flags(c, c->f[VFGPU_FIELD_U]);
  if (e == cudaSuccess) {
    if (precision == VFGPU_FP64) {
      e = launch_u_apply<double>(u_args<double>(c, xd, c->f[VFGPU_FIELD_V], yd, c->seam64, c->plan64),
                                 c->plan64, c->layers, c->stream);
    } else {
      int st = ensure_v32(c);
      if (st) return st;
      e = convert_f64_f32(xd, c->t32a, n3, c->stream);
      if (e == cudaSuccess)
        e = launch_u_apply<float>(u_args<float>(c, c->t32a, c->V32, c->t32b, c->seam32, c->plan32),
                                  c->plan32, c->layers, c->stream);
      if (e == cudaSuccess) e = convert_f32_f64(c->t32b, yd, n3, c->stream);
    }
  }
  if (e == cudaSuccess && !ydev) e = copy_out(c, y, yd, n3);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply");
  return VFGPU_OK;
}

int vfgpu_u_apply_dev(vfgpu_ctx* c, int precision, const void* x, void* y) {
  if (!c || !x || !y) return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_dev: null argument");
  if (precision != VFGPU_FP64 && precision != VFGPU_MIXED)
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_dev: bad precision %d", precision);
  if (!c->have_mat) return fail(VFGPU_ERR_STATE, "vfgpu_u_apply_dev: material not set");
  if (!is_device_ptr(x) || !is_device_ptr(y))
    return fail(VFGPU_ERR_INVALID, "vfgpu_u_apply_dev: x and y must be device pointers");
  cudaSetDevice(c->dev);
  cudaError_t e = u_lists_refresh(c);
  if (e == cudaSuccess && c->unilateral) e = nc_flags(c, c->f[VFGPU_FIELD_U]);
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_dev");
  if (precision == VFGPU_FP64) {
    e = launch_u_apply<double>(u_args<double>(c, (const double*)x, c->f[VFGPU_FIELD_V], (double*)y,
                                              c->seam64, c->plan64),
                               c->plan64, c->layers, c->stream);
  } else {
    int st = ensure_v32(c);
    if (st) return st;
    e = launch_u_apply<float>(u_args<float>(c, (const float*)x, c->V32, (float*)y, c->seam32,
                                            c->plan32),
                              c->plan32, c->layers, c->stream);
  }
  if (e != cudaSuccess) return cuda_fail(e, "vfgpu_u_apply_dev");
  return VFGPU_OK;
}

int vfgpu_get_stream(vfgpu_ctx* c, void** stream) {
  if (!c || !stream) return fail(VFGPU_ERR_INVALID, "vfgpu_get_stream: null argument");
  *stream = (void*)c->stream;
  return VFGPU_OK;
}

}  // extern "C"
