// Mixed-precision LU + FP64 refinement: placeholder until the tensor-core factorisation lands.
#include <stdexcept>

#include "mixed.h"

namespace bgpu {

struct MixedSolver::Impl {};

MixedSolver::MixedSolver() : p_(new Impl) {}
MixedSolver::~MixedSolver() { delete p_; }
const char* MixedSolver::name() const { return "mixed"; }
void MixedSolver::build(const DevMesh&, const DevDeflation&, double*, long, double, cudaStream_t, cudaEvent_t,
                        cudaEvent_t) {
  throw std::runtime_error("the mixed-precision factorisation is not available in this build (use fp64)");
}
void MixedSolver::solve(int, double*, long, cudaStream_t, MixedReport*) {
  throw std::runtime_error("the mixed-precision solve is not available in this build");
}

}  // namespace bgpu
