// ORACLE (test infrastructure only).  A C wrapper around the reference's own bit-exact C++ port of
// TGETGR/triangleint (hmatrix/src/kernel.cpp, bh::Kernel), so that tests and the CPU baseline can
// call the reference's assembly through ctypes.  It is compiled together with that file, from the
// reference tree, into oracle/_ref/ by oracle/Makefile; the reference's sources are never copied.
//
// Calls: bh::mesh_from_best (kernel.cpp:36-52), bh::Kernel::Kernel (kernel.cpp:54-146),
// Kernel::fill (kernel.cpp:262-275), Kernel::x, Kernel::diag_mean (kernel.cpp:278-286).
#include <memory>
#include <vector>

#include "kernel.h"

namespace {
std::unique_ptr<bh::Mesh> g_mesh;
std::unique_ptr<bh::Kernel> g_kernel;
}  // namespace

extern "C" {

// Sets up the reference kernel for a mesh in BEST's layout (n x 3 column-major, centred,
// corrected areas).  Returns 0.
int ref_create(int n, const double* v1, const double* v2, const double* v3, const double* area, double afac,
               double cg) {
  g_kernel.reset();
  g_mesh = std::make_unique<bh::Mesh>(bh::mesh_from_best(n, v1, v2, v3, area, afac));
  g_kernel = std::make_unique<bh::Kernel>(*g_mesh, cg);
  return 0;
}

// Incenters, n x 3 column-major.
void ref_incenters(double* x) {
  const int n = g_kernel->n();
  const std::vector<double>& xc = g_kernel->x();
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) x[size_t(c) * n + i] = xc[3 * size_t(i) + c];
}

// GR for target triangles [r0, r1) x source triangles [c0, c1), column-major with leading
// dimension lda, threaded over source columns with OpenMP.
void ref_fill(int r0, int r1, int c0, int c1, double* a, long lda) {
  const int m = r1 - r0, nc = c1 - c0;
  std::vector<int> rt(m);
  for (int i = 0; i < m; ++i) rt[i] = r0 + i;
#pragma omp parallel for schedule(dynamic, 8)
  for (int j = 0; j < nc; ++j) {
    const int ct = c0 + j;
    g_kernel->fill(rt.data(), m, &ct, 1, a + size_t(3 * j) * lda, int(lda));
  }
}

double ref_diag_mean(void) { return g_kernel->diag_mean(); }

void ref_destroy(void) {
  g_kernel.reset();
  g_mesh.reset();
}
}
