// Mixed-precision factorisation and refined solve (internal interface of libbestgpu).
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "bgpu_internal.h"

namespace bgpu {

// The mixed path cannot deliver (zero pivot without pivoting, refinement not converging): the caller
// falls back to the FP64 LU of the kept FP64 matrix.
struct MixedFailure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct MixedReport {
  int iterations = 0;   // refinement steps of the last solve
  double relres = 0.0;  // largest relative residual ||b - A x|| / ||b|| over the right-hand sides
};

// The mixed LU's diagonal leaf on one h x h block (h <= 128) of A (column-major, lda): LU without
// pivoting in place, L^-1 into DL and U^-1 into DU (128 x 128 column-major each, zero outside h x h).
// A zero or non-finite pivot sets *status to a nonzero code.
cudaError_t lu32_leaf(float* A, long lda, int h, float* DL, float* DU, int* status, cudaStream_t s);

class MixedSolver {
 public:
  MixedSolver();
  ~MixedSolver();
  MixedSolver(const MixedSolver&) = delete;
  MixedSolver& operator=(const MixedSolver&) = delete;
  const char* name() const;
  // Assembles GR + deflation into gr64 (FP64, kept for the residuals) and a reduced-precision copy,
  // records ev_assembled, factors the copy.  Throws on failure.  wait = false: returns once the work
  // is enqueued on s (other solvers' builds may then run beside it); finish_build(s) completes it.
  void build(const DevMesh& m, const DevDeflation& d, double* gr64, long ld, double eps, cudaStream_t s,
             cudaEvent_t ev_assembled, cudaEvent_t ev_factored, bool wait = true);
  // Waits for the factorisation enqueued on s, checks its status (throws MixedFailure).
  void finish_build(cudaStream_t s);
  // With BEST_GPU_PROFILE=1: per-category times of the calls since the last report (log lines).
  std::vector<std::string> profile_report();
  // GMRES restarts (each with a true FP64 residual) and Krylov vectors per restart.
  void set_refinement(int max_restarts, int krylov);
  // Solves GR x = b in place (d_b: 3n x nrhs, ldb) to the relative residual of build's eps.
  void solve(int nrhs, double* d_b, long ldb, cudaStream_t s, MixedReport* rep);
  // Device memory the solver holds (its factor, mirrors, inverses and scratch), reused by the next build.
  size_t device_bytes() const;

 private:
  struct Impl;
  Impl* p_;
};

}  // namespace bgpu
