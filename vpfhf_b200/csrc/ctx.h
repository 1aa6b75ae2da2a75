// ctx.h -- the resident problem state behind a vfgpu_ctx handle.
#pragma once

#include <string>
#include <vector>

#include "../../include/vfgpu.h"
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
  float* d_cellE = nullptr;     // NC or null
  bool have_mat = false;
  vfgpu_vfprop vf{0.2, 1e-5, 5e-2, 2, 0};  // VFPropGet defaults (VFCommon.c:468-480)

  // BCs
  vfgpu_bc bcU[3]{}, bcV{};
  uint8_t* bcU_kind = nullptr;  // 3N: VFGPU_BC_* per dof
  uint8_t* bcU_bits = nullptr;  // N: bit c => dof (n,c) Dirichlet
  uint8_t* bcV_kind = nullptr;  // N
  uint8_t* bcV_bits = nullptr;  // N: bit 0

  // fields (FP64, resident)
  double* f[7] = {nullptr};
  float* V32 = nullptr;  // FP32 copy of V for the mixed-precision operator
  bool v32_stale = true;

  // scratch
  vfgpu::UPlan plan64{}, plan32{};
  double* seam64 = nullptr;
  float* seam32 = nullptr;
  double *t64a = nullptr, *t64b = nullptr;
  float *t32a = nullptr, *t32b = nullptr;
};

namespace vfgpu {
int64_t field_len(const vfgpu_ctx* c, int field);
}
