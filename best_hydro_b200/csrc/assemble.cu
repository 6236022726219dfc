// Assembly of BEST's boundary-element matrix GR on the B200 (FP64).
//
// Compiled with -fmad=false: BEST is built with -ffp-contract=off (reference Makefile:34, :40), so
// every product and sum below must round separately, in the order the reference writes it, for the
// entries to follow the reference's operation sequence exactly.  IEEE +, -, *, / and sqrt are
// correctly rounded on both sides; every transcendental function (acos, sin, cos, log of the O(N)
// self blocks, and the 21 logs of each pair integral) is the correctly rounded one of ddmath.cuh.
// The entries therefore equal TGETGR's arithmetic with correctly rounded functions bit for bit.
// glibc's log, which the reference calls, is not correctly rounded on about 0.15 % of arguments, so
// about 0.06 % of the reference's entries differ from these by an ulp or a few; each such entry is
// one whose pair meets such an argument.
//
// Kernels:
//   k_self_blocks   one thread per triangle: incenter, normal and the exact self-integral block,
//                   best/tgetgr.f:33-147 (the C++ twin is hmatrix/src/kernel.cpp:54-146)
//   k_assemble      one thread per (target, source) pair, targets along threadIdx.x so each warp's
//                   stores of a column are contiguous; the source triangles of a tile are staged in
//                   shared memory with their target-independent differences and dot products.
//                   best/triangleint.f:1-247 (kernel.cpp:148-249); epilogue: the deflation term of
//                   best/best.f:406-425 and an optional FP32 copy for the mixed-precision LU.
//   k_assemble_series  the same tiles for every mesh of a series (up to 16) in one launch
//   k_diag_mean     best/best.f:401-403, summed in BEST's order (one thread: the order is the spec).
#include <cuda_runtime.h>

#include "assemble_tile.cuh"
#include "bgpu_internal.h"
#include "ddmath.cuh"

namespace bgpu {
namespace {

constexpr double kPi = 3.1415926535897932385;  // tgetgr.f:17
using dd::cr_acos;
using dd::cr_cos;
using dd::cr_log;
using dd::cr_sin;

// tgetgr.f:177-187
__device__ __forceinline__ double si_fn(double x) {
  return 2.0 * (cr_log((1.0 + sqrt(1.0 - x * x)) / x) - sqrt(1.0 - x * x));
}
__device__ __forceinline__ double csi_fn(double x) { return 3.0 - 1.0 / x - 2.0 * x; }

__global__ void k_self_blocks(int n, const double* __restrict__ geo, double afac, double cg, double* __restrict__ xc,
                              double* __restrict__ self9) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double* g = geo + (size_t)t * kGeoStride;
  const double p1x = g[0], p1y = g[1], p1z = g[2];
  const double p2x = g[3], p2y = g[4], p2z = g[5];
  const double p3x = g[6], p3y = g[7], p3z = g[8];
  const double pi = kPi;
  // incenter (tgetgr.f:36-52)
  const double v21x = p2x - p1x, v21y = p2y - p1y, v21z = p2z - p1z;
  const double v31x = p3x - p1x, v31y = p3y - p1y, v31z = p3z - p1z;
  const double v32x = p3x - p2x, v32y = p3y - p2y, v32z = p3z - p2z;
  const double a = sqrt(v21x * v21x + v21y * v21y + v21z * v21z);
  const double b = sqrt(v31x * v31x + v31y * v31y + v31z * v31z);
  const double c = sqrt(v32x * v32x + v32y * v32y + v32z * v32z);
  const double cosC = (v21x * v31x + v21y * v31y + v21z * v31z) / a / b;
  const double tin = (a + b - c) / (2. * (1. + cosC));
  xc[(size_t)t * kXcStride + 0] = p1x + tin * (v21x / a + v31x / b);
  xc[(size_t)t * kXcStride + 1] = p1y + tin * (v21y / a + v31y / b);
  xc[(size_t)t * kXcStride + 2] = p1z + tin * (v21z / a + v31z / b);
  xc[(size_t)t * kXcStride + 3] = 0.0;
  // unit normal (:56-63)
  double nx = v31y * v21z - v31z * v21y;
  double ny = v31z * v21x - v31x * v21z;
  double nz = v31x * v21y - v31y * v21x;
  const double area2 = sqrt(nx * nx + ny * ny + nz * nz) / 2.;
  nx = .5 * nx / area2;
  ny = .5 * ny / area2;
  nz = .5 * nz / area2;
  // exact self integrals (:67-112)
  const double cc = cr_acos(cosC);
  const double r = tin * cr_sin(cc);
  const double cosB = -(v21x * v32x + v21y * v32y + v21z * v32z) / a / c;
  const double bb = cr_acos(cosB);
  const double aa = pi - bb - cc;
  const double hcos = 1. / (2. * cr_cos(0.5 * cc));
  const double dc = (a + b - c) * hcos;
  const double db = sqrt(a * a + (b - c) * (b - c) - 2. * a * (b - c) * cosC) * hcos;
  const double da = sqrt(b * b + (a - c) * (a - c) - 2. * b * (a - c) * cosC) * hcos;
  const double ha = r / da, hb = r / db, hc = r / dc;
  const double dpa = (pi - aa) * (da - r) - 2.0 * (da * cr_acos(ha) - r * cr_log((1. + sqrt(1. - ha * ha)) / ha));
  const double dpb = (pi - bb) * (db - r) - 2.0 * (db * cr_acos(hb) - r * cr_log((1. + sqrt(1. - hb * hb)) / hb));
  const double dpc = (pi - cc) * (dc - r) - 2.0 * (dc * cr_acos(hc) - r * cr_log((1. + sqrt(1. - hc * hc)) / hc));
  const double sca =
      0.5 * r * ((cr_cos(2.0 * cc) + cr_cos(2.0 * bb)) * si_fn(ha) - (cr_sin(2.0 * cc) + cr_sin(2.0 * bb)) * csi_fn(ha));
  const double scb = 0.5 * r * ((1. + cr_cos(2.0 * bb)) * si_fn(hb) + cr_sin(2.0 * bb) * csi_fn(hb));
  const double scc = 0.5 * r * ((1. + cr_cos(2.0 * cc)) * si_fn(hc) + cr_sin(2.0 * cc) * csi_fn(hc));
  const double cca = -(cr_sin(bb - cc) * r * (cr_cos(aa) * si_fn(ha) + cr_sin(aa) * csi_fn(ha)));
  const double ccb = cr_sin(bb) * r * (cr_cos(bb) * si_fn(hb) + cr_sin(bb) * csi_fn(hb));
  const double ccc = -(cr_sin(cc) * r * (cr_cos(cc) * si_fn(hc) + cr_sin(cc) * csi_fn(hc)));
  const double cor = sqrt(afac);
  // local g (1-based as in the Fortran; g(1,3) = g(2,3) = g(3,1) = g(3,2) = 0)
  double gl[4][4];
  gl[1][1] = cor * ((2.0 + cg) * pi * r + (1.0 + 0.5 * cg) * cg * (dpa + dpb + dpc) + cg * 0.25 * (sca + scb + scc));
  gl[1][2] = 0.5 * cor * (cca + ccb + ccc) * cg;
  gl[2][1] = gl[1][2];
  gl[2][2] = gl[1][1] - 0.5 * cor * cg * (sca + scb + scc);
  gl[3][3] = cor * (2.0 * pi * r + (dpa + dpb + dpc));
  gl[1][3] = gl[2][3] = gl[3][1] = gl[3][2] = 0.0;
  // rotation to the lab frame (:121-145)
  double rr[4][4];
  rr[1][1] = v21x / a;
  rr[1][2] = v21y / a;
  rr[1][3] = v21z / a;
  rr[3][1] = nx;
  rr[3][2] = ny;
  rr[3][3] = nz;
  rr[2][1] = (ny * v21z - nz * v21y) / a;
  rr[2][2] = (nz * v21x - nx * v21z) / a;
  rr[2][3] = (nx * v21y - ny * v21x) / a;
  double* out = self9 + (size_t)t * 9;
#pragma unroll
  for (int i = 1; i <= 3; ++i)
#pragma unroll
    for (int j = 1; j <= 3; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int k = 1; k <= 3; ++k)
        acc = acc + rr[k][i] * (gl[k][1] * rr[1][j] + gl[k][2] * rr[2][j] + gl[k][3] * rr[3][j]);
      out[3 * (i - 1) + (j - 1)] = acc;
    }
}

__global__ void __launch_bounds__(kTgtTile, BGPU_ASM_MIN_BLOCKS)
    k_assemble(const double* __restrict__ geo, const double* __restrict__ xc, const double* __restrict__ self9,
               double cg, int r0, int r1, int c0, int c1, double* __restrict__ out, long ld, DevDeflation defl,
               float* __restrict__ out32, long ld32) {
  __shared__ double s_logtab[3 * dd::kLogTabN];
  assemble_tile<false>(blockIdx.x, blockIdx.y, geo, xc, self9, cg, r0, r1, c0, c1, out, ld, defl, out32, ld32,
                       s_logtab);
}

// Every mesh of a series in one launch: block b belongs to the mesh whose tile range holds it.
__global__ void __launch_bounds__(kTgtTile, BGPU_ASM_MIN_BLOCKS) k_assemble_series(const __grid_constant__ SeriesAssembly sa) {
  const int b = blockIdx.x;
  int i = 0;
  while (i + 1 < sa.count && b >= sa.tile0[i + 1]) ++i;
  const int local = b - sa.tile0[i];
  const int tx = (sa.mesh[i].n + kTgtTile - 1) / kTgtTile;
  const DevMesh& m = sa.mesh[i];
  __shared__ double s_logtab[3 * dd::kLogTabN];
  assemble_tile<false>(local % tx, local / tx, m.geo, m.xc, m.self9, m.cg, 0, m.n, 0, m.n, sa.out[i], sa.ld[i], sa.defl[i],
                       nullptr, 0, s_logtab);
}

__global__ void k_diag_mean(int n, const double* __restrict__ self9, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int t = 0; t < n; ++t) s = s + self9[9 * (size_t)t] + self9[9 * (size_t)t + 4] + self9[9 * (size_t)t + 8];
  *out = s / (double)(3 * n);
}

}  // namespace

cudaError_t launch_self_blocks(const DevMesh& m, cudaStream_t s) {
  if (m.n <= 0) return cudaSuccess;
  k_self_blocks<<<(m.n + 127) / 128, 128, 0, s>>>(m.n, m.geo, m.afac, m.cg, m.xc, m.self9);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_assemble(const DevMesh& m, int r0, int r1, int c0, int c1, double* out, long ld,
                            const DevDeflation& defl, float* out32, long ld32, cudaStream_t s) {
  if (r1 <= r0 || c1 <= c0) return cudaSuccess;
  dim3 grid((r1 - r0 + kTgtTile - 1) / kTgtTile, (c1 - c0 + kSrcTile - 1) / kSrcTile);
  if (grid.y > 65535u) {
    // more source tiles than one grid dimension holds: split along the sources
    const int chunk = 65535 * kSrcTile;
    for (int c = c0; c < c1; c += chunk) {
      cudaError_t e = launch_assemble(m, r0, r1, c, c + (c1 - c < chunk ? c1 - c : chunk), out + 3 * (size_t)(c - c0) * ld,
                                      ld, defl, out32 ? out32 + 3 * (size_t)(c - c0) * ld32 : nullptr, ld32, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  k_assemble<<<grid, kTgtTile, 0, s>>>(m.geo, m.xc, m.self9, m.cg, r0, r1, c0, c1, out, ld, defl, out32, ld32);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_assemble_series(const SeriesAssembly& sa, cudaStream_t s) {
  if (sa.count <= 0) return cudaSuccess;
  SeriesAssembly a = sa;
  long total = 0;
  for (int i = 0; i < a.count; ++i) {
    a.tile0[i] = (int)total;
    const long tx = (a.mesh[i].n + kTgtTile - 1) / kTgtTile, ty = (a.mesh[i].n + kSrcTile - 1) / kSrcTile;
    total += tx * ty;
  }
  if (total > 0x7fffffffL) return cudaErrorInvalidValue;
  k_assemble_series<<<(unsigned)total, kTgtTile, 0, s>>>(a);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_diag_mean(const DevMesh& m, double* d_out, cudaStream_t s) {
  k_diag_mean<<<1, 32, 0, s>>>(m.n, m.self9, d_out);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace bgpu
