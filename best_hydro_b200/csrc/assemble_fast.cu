// GR assembly for the mixed-precision path: the pair integrals of best/triangleint.f with fewer FP64
// operations (assemble_tile<true>: rsqrt for 1/sqrt, shared reciprocals, the hy/hxy/hx denominators
// as quadratics in y), compiled with FMA contraction.  Entries agree with the bit-exact kernel to a
// few ulp; the mixed path's accuracy bar is on D_t, D_r, [eta] at 1e-8, which its FP64 refinement
// against this same matrix meets.  Self blocks, deflation and the FP32 copy as the exact kernel.
#include <cuda_runtime.h>

#include "assemble_tile.cuh"
#include "bgpu_internal.h"

namespace bgpu {
namespace {

#ifndef BGPU_ASM_FAST_MIN_BLOCKS
#define BGPU_ASM_FAST_MIN_BLOCKS 4
#endif

__global__ void __launch_bounds__(kTgtTile, BGPU_ASM_FAST_MIN_BLOCKS)
    k_assemble_fast(const double* __restrict__ geo, const double* __restrict__ xc, const double* __restrict__ self9,
                    double cg, int r0, int r1, int c0, int c1, double* __restrict__ out, long ld, DevDeflation defl,
                    float* __restrict__ out32, long ld32) {
  assemble_tile<true>(blockIdx.x, blockIdx.y, geo, xc, self9, cg, r0, r1, c0, c1, out, ld, defl, out32, ld32, nullptr);
}

}  // namespace

cudaError_t launch_assemble_fast(const DevMesh& m, int r0, int r1, int c0, int c1, double* out, long ld,
                                 const DevDeflation& defl, float* out32, long ld32, cudaStream_t s) {
  if (r1 <= r0 || c1 <= c0) return cudaSuccess;
  if (!m.fast_ok) return launch_assemble(m, r0, r1, c0, c1, out, ld, defl, out32, ld32, s);
  dim3 grid((r1 - r0 + kTgtTile - 1) / kTgtTile, (c1 - c0 + kSrcTile - 1) / kSrcTile);
  if (grid.y > 65535u) {
    // more source tiles than one grid dimension holds: split along the sources
    const int chunk = 65535 * kSrcTile;
    for (int c = c0; c < c1; c += chunk) {
      cudaError_t e = launch_assemble_fast(m, r0, r1, c, c + (c1 - c < chunk ? c1 - c : chunk),
                                           out + 3 * (size_t)(c - c0) * ld, ld, defl,
                                           out32 ? out32 + 3 * (size_t)(c - c0) * ld32 : nullptr, ld32, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  k_assemble_fast<<<grid, kTgtTile, 0, s>>>(m.geo, m.xc, m.self9, m.cg, r0, r1, c0, c1, out, ld, defl, out32, ld32);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace bgpu
