// cg.cuh -- preconditioned CG with device-resident scalars (no host round trip per
// iteration) and deterministic reductions.
//
// Semantics of PETSc's KSPCG with KSP_NORM_PRECONDITIONED and the default
// convergence test (KSPConvergedDefault): x0 = 0, z = D^-1 r, converged when
// ||z|| <= max(rtol ||z0||, atol), diverged on ||z|| >= dtol ||z0||, NaN, or a
// non-positive p.Ap.  Vectors are T (double, or float for the inner solve of the
// mixed-precision path); every dot product and step length is FP64.
#pragma once

#include "common.cuh"

namespace vfgpu {

// Reason codes (PETSc KSPConvergedReason numbering where one exists).
enum { CG_RUNNING = 0, CG_CONVERGED_RTOL = 2, CG_CONVERGED_ATOL = 3, CG_DIVERGED_ITS = -3,
       CG_DIVERGED_DTOL = -4, CG_DIVERGED_INDEFINITE = -8, CG_DIVERGED_NAN = -9 };

struct CGState {
  double rz, rz_new, pw, zz, alpha, beta, rnorm0, ttol, dtol;
  double xalpha;  // step of the current iteration (0 if it made none); see cg_after_apply
  int its, maxit, done, reason;
  unsigned int arrive;  // blocks of the running update kernel that have finished
};

// Fixed reduction grid (4 blocks per SM of a B200): the block partials are summed in
// a fixed order, so every reduction is deterministic.
constexpr int RED_THREADS = 256, RED_BLOCKS = 592;

// The vectors are whole device allocations (16-byte aligned: the kernels use 16-byte
// loads and stores).
template <typename T> struct CGVecs {
  T* x;              // solution
  T* r;              // residual
  T* p;              // search direction
  T* w;              // A p
  const T* dinv;     // Jacobi: 1 / diag
  const T* b;        // right-hand side
  const uint8_t* mask;  // nonzero => dof removed from the system (or null)
  int64_t n;
  const double* dotp;   // the operator's block partials of p.w (written by the apply), or
  int ndot;             // null: cg_after_apply computes p.w in a separate pass
};

// Host-side driver pieces (solver.cu).  One iteration is: the operator apply
// w = A p, which also writes the block partials of p.w to v.dotp (the tile
// engine's A.dot), then cg_after_apply: the update kernel moves r only (r -= alpha w,
// z = D^-1 r, (r,z), (z,z)), and the direction kernel does x += alpha p together with
// p = z + beta p, in one pass over p.  The iteration that stops the solve skips the
// direction kernel, so cg_finish_x adds its step to x after the loop.
template <typename T>
cudaError_t cg_init(const CGVecs<T>& v, CGState* st, double* partial, double rtol, double atol,
                    double dtol, int maxit, cudaStream_t s);
template <typename T>
cudaError_t cg_after_apply(const CGVecs<T>& v, CGState* st, double* partial, cudaStream_t s);
template <typename T>
cudaError_t cg_finish_x(const CGVecs<T>& v, const CGState* st, cudaStream_t s);

}  // namespace vfgpu
