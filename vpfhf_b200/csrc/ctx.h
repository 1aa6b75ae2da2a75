// ctx.h -- the resident problem state behind a vfgpu_ctx handle.
#pragma once

#include <string>
#include <vector>

#include "../../include/vfgpu.h"
#include "cg.cuh"
#include "elem.h"
#include "kernels.h"

struct vfgpu_ctx {
  int dev = 0, nsm = 148;
  int nx = 0, ny = 0, nz = 0;
  double lx = 0, ly = 0, lz = 0, hx = 0, hy = 0, hz = 0;
  int64_t N = 0;   // nodes
  int64_t NC = 0;  // cells
  cudaStream_t stream = nullptr;

  // material
  int nlayer = 0;
  vfgpu::LayerTable layers{};
  uint8_t* d_elayer = nullptr;  // nz-1
  // U unit lists of plan64 / plan32 (UnitLists::cls null: the grid takes none), in one
  // allocation; rebuilt from the FP64 v by u_lists_refresh when ul_stale (set with
  // v32_stale wherever v changes)
  void* d_ul = nullptr;
  vfgpu::UnitLists ul64, ul32;
  bool ul_stale = true;
  int u_split = VFGPU_U_SPLIT_AUTO;
  vfgpu::DevParams* d_params = nullptr;  // device copy of layers / eta / aeps
  float* d_cellE = nullptr;     // NC or null
  bool have_mat = false;
  vfgpu_vfprop vf{0.2, 1e-5, 5e-2, 2, 0};  // VFPropGet defaults (VFCommon.c:468-480)

  // unilateral model (VFCtx.unilateral): 1 = NOCOMPRESSION, with the per-cell
  // compression bits of the current linearisation point
  int unilateral = 0;
  uint32_t* d_cflag = nullptr;  // NC
  void* d_tcB = nullptr;        // tensor-core apply: its constant operands (tc_apply.cu)
  unsigned* d_tcerr = nullptr;  // tensor-core apply: bounded-wait flag

  // in-situ stresses (VFCtx.hasInsitu, insitumin, insitumax)
  bool has_insitu = false;
  double insitu_min[6]{}, insitu_max[6]{};

  // BCs
  vfgpu_bc bcU[3]{}, bcV{};
  uint8_t* bcU_kind = nullptr;  // 3N: VFGPU_BC_* per dof
  uint8_t* bcU_bits = nullptr;  // N: bit c => dof (n,c) Dirichlet
  uint8_t* bcV_kind = nullptr;  // N
  uint8_t* bcV_bits = nullptr;  // N: bit 0

  // fields (FP64, resident)
  double* f[7] = {nullptr};
  float* V32 = nullptr;  // FP32 copy of V for the mixed-precision operator
  bool v32_stale = true;  // (with ul_stale)

  // scratch
  vfgpu::TilePlan plan64{}, plan32{}, vplan64{}, vplan32{};
  double* d_dot = nullptr;   // block partials of the CG's p.w written by the operator applies
  double* seam64 = nullptr;  // U and V seams FP64 (sized for the larger of the two plans)
  float* seam32 = nullptr;
  double *t64a = nullptr, *t64b = nullptr;
  float *t32a = nullptr, *t32b = nullptr;

  // solver work space, allocated at the first solve (see solve_buffers in step.cu)
  static constexpr int NP64 = 9, NP32 = 5;
  double* p64[NP64] = {nullptr};  // 3N + kPoolSlack doubles each
  float* p32[NP32] = {nullptr};   // 3N + kPoolSlack floats each
  double* coef64 = nullptr;       // 27 per cell: V coupling coefficient (vcoef_index layout)
  float* coef32 = nullptr;
  CUtensorMap vmap64{}, vmap32{}; // coef64 / coef32 as the V apply's tensor copies see them
  unsigned* d_cerr = nullptr;     // set by an apply whose bounded wait on a tensor copy (V
                                  // coefficients, U node planes) gave up; held for the ctx's life
  uint8_t* vmask = nullptr;       // N
  vfgpu::ETab h_tab{};            // element tables of the uniform element (kernel parameter)
  vfgpu::CGState* d_cg = nullptr; // device CG scalars
  vfgpu::CGState* h_cg = nullptr; // pinned host mirror
  double* d_red = nullptr;        // reduction partials (RED_BLOCKS * 4 + energy blocks * 4)
  double* d_out = nullptr;        // small device results (16 doubles)
  double* h_out = nullptr;        // pinned host mirror of d_out
  bool have_solver = false;

  // Geometric multigrid hierarchy of the U operator (VFGPU_PC_MG), built at the first
  // MG solve in the V-cycle's precision (mg_bytes: 8 FP64, 4 FP32): level 0 is the
  // ctx's own grid (work vectors only), levels 1.. halve the cells per axis.
  struct MGLevel {
    int nx = 0, ny = 0, nz = 0;
    int64_t N = 0, NC = 0;
    double hx = 0, hy = 0, hz = 0;
    vfgpu::TilePlan plan{};
    void* seam = nullptr;                      // V-cycle precision
    void *x = nullptr, *b = nullptr, *r = nullptr, *d = nullptr, *t = nullptr;  // 3N each
    void* ev = nullptr;                        // 3N: the power iteration's vector, kept
    void *v = nullptr, *dinv = nullptr;        // coarse phase field (N), inverse diagonal (3N)
    double* v64 = nullptr;                     // coarse phase field in FP64 (the diagonal's input)
    uint8_t *bc = nullptr, *elayer = nullptr;
    float* cellE = nullptr;
    int* xi = nullptr;     // transfer from the finer level: pI (x, y, z), rlo (x, y, z), rn (x, y, z)
    double* xw = nullptr;  // pw (x, y, z)
    vfgpu::ETab tab{};
    double* coef = nullptr;  // device, 64: lmax, 1/theta, Chebyshev (c1, c2) pairs, scratch
  };
  std::vector<MGLevel> mg;
  int mg_bytes = 0;
  bool mg_ready = false;          // coarse fields, diagonals and eigenvalue bounds are current
  bool mg_ev = false;             // the levels' ev vectors hold earlier eigenvector estimates
  bool mg_layers = false;         // the coarse levels' element layers match d_elayer
  double* mg_coef = nullptr;      // 64 doubles per level (MGLevel::coef points into it)
  double* mg_z = nullptr;         // FP32 V-cycle: the preconditioned residual in FP64 (3N)
  const void* mg_dinv0 = nullptr; // fine inverse diagonal in the V-cycle's precision

  // Flow-coupling boundary (width.cu): cell width, permeability multiplier, node width,
  // stalled-march count, well-rate scratch; allocated at the first width call.
  double *d_widthc = nullptr, *d_pmult = nullptr, *d_width = nullptr, *d_wpart = nullptr;
  unsigned* d_wstall = nullptr;

  // Host-buffer apply pipeline (vfgpu_u_apply with host x and y): a second output
  // staging vector, the copy streams and one event per slab, made at the first use.
  static constexpr int kPipeSlabs = 16;
  double* t64c = nullptr;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_start = nullptr, ev_in[kPipeSlabs] = {}, ev_y[kPipeSlabs] = {},
              ev_out[kPipeSlabs] = {};

  // Captured CUDA graphs of CG iteration batches, keyed by (call site, batch size).
  // Kernels read the material table, eta and the AT gradient weights through
  // d_params, so new material / vfprop values leave the graphs valid; a set-up call
  // that changes a captured pointer (the cell-modulus array) bumps `gen` and stale
  // graphs are re-captured.
  struct Graph {
    int kind, batch;
    uint64_t gen;
    cudaGraphExec_t exec;
  };
  std::vector<Graph> graphs;
  uint64_t gen = 1;
  bool use_graphs = true;
  // per CG call site (run_cg kind 1..4): iterations of its last solve, the size of
  // the first batch of the next one
  int cg_last_its[8] = {0};
};

namespace vfgpu {
int64_t field_len(const vfgpu_ctx* c, int field);
// Solver pools hold 3N + kPoolSlack values; N-vectors carved from them start at
// multiples of pool_stride(N) (a multiple of 4 values: 16-byte aligned for float
// and double).
constexpr int64_t kPoolSlack = 16;
inline int64_t pool_stride(int64_t n) { return (n + 3) & ~int64_t(3); }
}
