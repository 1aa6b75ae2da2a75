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
  double xalpha;  // step of the solution update still to be applied (0: none)
  int its, maxit, done, reason;
  unsigned int arrive;  // blocks of the running update kernel that have finished
};

// Fixed reduction grid (4 blocks per SM of a B200): the block partials are summed in
// a fixed order, so every reduction is deterministic.
constexpr int RED_THREADS = 256, RED_BLOCKS = 592;

// The vectors are whole device allocations (16-byte aligned: the kernels use 16-byte
// loads and stores).
// With p2 non-null the solution update is fused into the operator apply: iteration i
// applies the operator to p_i (buffer i % 2: p, p2) and the apply also adds
// xalpha p_{i-1} (the other buffer) to x for every node it finishes; the update kernel
// then moves only r, and the direction update writes p_{i+1} into the other buffer.
// After the last iteration cg_finish_x adds the pending step.  Iteration parity follows
// the global iteration count, so batches of iterations must be even.  With p2 null
// (one direction buffer) the update kernel updates x itself.
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
  T* p2 = nullptr;      // second direction buffer: fused solution update (see above)
  T* pcur(int parity) const { return (p2 && (parity & 1)) ? p2 : p; }
  T* pother(int parity) const { return p2 ? ((parity & 1) ? p : p2) : p; }
};

// Host-side driver pieces (solver.cu).  One iteration is: the operator apply
// w = A p, which also writes the block partials of p.w to v.dotp (the tile
// engine's A.dot), then cg_after_apply.
template <typename T>
cudaError_t cg_init(const CGVecs<T>& v, CGState* st, double* partial, double rtol, double atol,
                    double dtol, int maxit, cudaStream_t s);
template <typename T>
cudaError_t cg_after_apply(const CGVecs<T>& v, CGState* st, double* partial, cudaStream_t s,
                           int parity = 0);
// Fused mode: x += xalpha p_last, the step of the last iteration (of parity `parity`).
template <typename T>
cudaError_t cg_finish_x(const CGVecs<T>& v, const CGState* st, int parity, cudaStream_t s);

}  // namespace vfgpu
