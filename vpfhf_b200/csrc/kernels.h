// kernels.h -- host-side declarations of the vfgpu kernel launchers.
#pragma once

#include <algorithm>

#include "common.cuh"
#include "ops.cuh"

namespace vfgpu {

cudaError_t apply_kernel_attributes();
TilePlan u_plan(int nx, int ny, int nz, int prec_bytes, int num_sms);
TilePlan v_plan(int nx, int ny, int nz, int prec_bytes, int num_sms);
// Element rows of a V tile: the y extent of the coefficient tensor copy's box.
constexpr int kVTileY = 8;
// The V coefficient array (vcoef_index layout, 8- or 4-byte values) as the 3-D tensor
// the V apply stages from: box 32 x kVTileY x 27.
cudaError_t vcoef_tensor_map(CUtensorMap* map, const void* coef, int bytes, int nex, int ney, int nez);
// The bounded mbarrier wait of the tensor-copy pipeline, alone: *timed_out = 1 when a
// wait on a phase that never completes (complete = 0) gave up after `cycles`.
cudaError_t wait_selftest(long long cycles, int complete, int* timed_out);

// The U operator's unit lists for one tile plan (UApplyArgs::ur): the per-(tile,
// element layer) constant-phase-field flags and the two lists built from them.
struct UnitLists {
  uint8_t* cls = nullptr;  // [ntx nty][nz - 1]; null: no lists for this plan
  int4* runs[2] = {};      // [ntx nty nz] each
  int* start[2] = {};      // [ncta0], [ncta]
  int* total = nullptr;    // [2]
};
// Device bytes of a plan's unit lists; 0 when the grid has more tile columns than the
// one-block list builder takes (its applies then split all units).
size_t unit_lists_bytes(const TilePlan& p, int nz);
UnitLists unit_lists_carve(void* base, const TilePlan& p, int nz);
// Whether the split measured faster than one wave at this plan's size in precision
// prec_bytes (8 or 4): the VFGPU_U_SPLIT_AUTO rule.
bool unit_lists_pay(const TilePlan& p, int nz, int prec_bytes);
// Rebuilds the lists from the FP64 phase field v (two launches on s).
cudaError_t build_unit_lists(const double* v, int nx, int ny, int nz, const TilePlan& p,
                             const UnitLists& L, cudaStream_t s);
template <typename T> void use_unit_lists(UApplyArgs<T>& A, const UnitLists& L) {
  for (int l = 0; l < 2; l++) {
    A.ur[l] = L.cls ? L.runs[l] : nullptr;
    A.ustart[l] = L.cls ? L.start[l] : nullptr;
  }
  A.utotal = L.cls ? L.total : nullptr;
}

template <typename T>
cudaError_t launch_u_apply(const UApplyArgs<T>& A, const TilePlan& p, const LayerTable& L,
                           cudaStream_t s);
template <typename T>
cudaError_t launch_v_apply(const VApplyArgs<T>& A, const TilePlan& p, const LayerTable& L,
                           cudaStream_t s);

}  // namespace vfgpu
