// Assembly of BEST's boundary-element matrix GR on the B200 (FP64).
//
// Compiled with -fmad=false: BEST is built with -ffp-contract=off (reference Makefile:34, :40), so
// every product and sum below must round separately, in the order the reference writes it, for the
// entries to match the reference's bit for bit.  IEEE +, -, *, / and sqrt are correctly rounded on
// both sides.  The transcendental functions of the O(N) self blocks (acos, sin, cos, log) are the
// correctly rounded ones of ddmath.cuh, which return what glibc returns for almost every argument;
// the pair integrals' log is CUDA's (within an ulp; it reaches the entries without cancellation).
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

#include "bgpu_internal.h"
#include "ddmath.cuh"

namespace bgpu {
namespace {

constexpr double kPi = 3.1415926535897932385;  // tgetgr.f:17
constexpr int kTgtTile = 128;                   // targets per block (threads)
#ifndef BGPU_ASM_MIN_BLOCKS
#define BGPU_ASM_MIN_BLOCKS 4                   // resident blocks per SM the register budget allows
#endif
constexpr int kSrcTile = 16;                    // source triangles per block

// 21-point Gauss-Legendre abscissae and weights on [0,1]: the decimal literals of
// best/triangleint.f:66-108 (the same doubles are required for bit-compatible entries).
__constant__ double c_gy[21] = {
    3.1239146898052499e-3, 1.6386580716846853e-2, 3.9950332924799586e-2, 7.3318317708341358e-2,
    0.1157800182621610,    0.1664305979012938,    0.2241905820563901,    0.2878289398962806,
    0.3559893415987995,    0.4272190729195525,    0.5,                   0.5727809270804476,
    0.6440106584012005,    0.7121710601037194,    0.7758094179436099,    0.8335694020987062,
    0.8842199817378390,    0.9266816822916586,    0.9600496670752004,    0.9836134192831531,
    0.9968760853101948};
__constant__ double c_gw[21] = {
    1.601722825777433e-2, 3.695378977085249e-2, 5.713442542685720e-2, 7.610011362837930e-2,
    9.344442345603390e-2, 0.1087972991671484,   0.1218314160537285,   0.1322689386333375,
    0.1398873947910731,   0.1445244039899701,   0.1460811336496904,   0.1445244039899701,
    0.1398873947910731,   0.1322689386333375,   0.1218314160537285,   0.1087972991671484,
    9.344442345603390e-2, 7.610011362837930e-2, 5.713442542685720e-2, 3.695378977085249e-2,
    1.601722825777433e-2};

__device__ __forceinline__ double dot3(double a0, double a1, double a2, double b0, double b1, double b2) {
  return a0 * b0 + a1 * b1 + a2 * b2;
}

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

// One tile: targets [r0 + 128 bx, +128) x sources [c0 + 16 by, +16) of one mesh.
__device__ __forceinline__ void assemble_tile(int bx, int by, const double* __restrict__ geo,
                                              const double* __restrict__ xc, const double* __restrict__ self9,
                                              double cg, int r0, int r1, int c0, int c1, double* __restrict__ out,
                                              long ld, const DevDeflation& defl, float* __restrict__ out32, long ld32) {
  __shared__ double s_p[kSrcTile][9];     // p1, p2, p3
  __shared__ double s_v[kSrcTile][9];     // v21, v31, v32
  __shared__ double s_d[kSrcTile][8];     // d2121 d2131 d2132 d3131 d3232 d3231 s21 area
  __shared__ int s_comp[kSrcTile];

  const int sbase = c0 + by * kSrcTile;
  const int ns = min(kSrcTile, c1 - sbase);
  if (threadIdx.x < ns) {
    const int t = sbase + threadIdx.x;
    const double* gp = geo + (size_t)t * kGeoStride;
    double p[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) p[q] = gp[q];
#pragma unroll
    for (int q = 0; q < 9; ++q) s_p[threadIdx.x][q] = p[q];
    double v21[3], v31[3], v32[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v21[c] = p[3 + c] - p[c];
      v31[c] = p[6 + c] - p[c];
      v32[c] = p[6 + c] - p[3 + c];
      s_v[threadIdx.x][c] = v21[c];
      s_v[threadIdx.x][3 + c] = v31[c];
      s_v[threadIdx.x][6 + c] = v32[c];
    }
    const double d2121 = dot3(v21[0], v21[1], v21[2], v21[0], v21[1], v21[2]);
    s_d[threadIdx.x][0] = d2121;
    s_d[threadIdx.x][1] = dot3(v21[0], v21[1], v21[2], v31[0], v31[1], v31[2]);
    s_d[threadIdx.x][2] = dot3(v21[0], v21[1], v21[2], v32[0], v32[1], v32[2]);
    s_d[threadIdx.x][3] = dot3(v31[0], v31[1], v31[2], v31[0], v31[1], v31[2]);
    s_d[threadIdx.x][4] = dot3(v32[0], v32[1], v32[2], v32[0], v32[1], v32[2]);
    s_d[threadIdx.x][5] = dot3(v32[0], v32[1], v32[2], v31[0], v31[1], v31[2]);
    s_d[threadIdx.x][6] = sqrt(d2121);
    s_d[threadIdx.x][7] = gp[9];
    s_comp[threadIdx.x] = (defl.ndef > 1) ? defl.comp[t] : 1;
  }
  __syncthreads();

  const int n1 = r0 + bx * kTgtTile + threadIdx.x;
  if (n1 >= r1) return;
  const double xcx = xc[(size_t)n1 * kXcStride + 0];
  const double xcy = xc[(size_t)n1 * kXcStride + 1];
  const double xcz = xc[(size_t)n1 * kXcStride + 2];
  const int comp1 = (defl.ndef > 1) ? defl.comp[n1] : 1;
  double xmu_i[3] = {0.0, 0.0, 0.0};
  if (defl.ndef > 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) xmu_i[a] = defl.xmu[3 * (size_t)n1 + a];
  }
  const size_t row0 = 3 * (size_t)(n1 - r0);

  for (int si = 0; si < ns; ++si) {
    const int n2 = sbase + si;
    double blk[9];
    if (n2 == n1) {
#pragma unroll
      for (int q = 0; q < 9; ++q) blk[q] = self9[(size_t)n1 * 9 + q];
    } else {
      const double* P = s_p[si];
      const double* V = s_v[si];
      const double* D = s_d[si];
      const double v21[3] = {V[0], V[1], V[2]};
      const double v31[3] = {V[3], V[4], V[5]};
      const double v32[3] = {V[6], V[7], V[8]};
      const double v1c[3] = {P[0] - xcx, P[1] - xcy, P[2] - xcz};
      const double v2c[3] = {P[3] - xcx, P[4] - xcy, P[5] - xcz};
      const double v3c[3] = {P[6] - xcx, P[7] - xcy, P[8] - xcz};
      const double d2121 = D[0], d2131 = D[1], d2132 = D[2], d3131 = D[3], d3232 = D[4], d3231 = D[5];
      const double s21 = D[6];
      const double d211c = dot3(v21[0], v21[1], v21[2], v1c[0], v1c[1], v1c[2]);
      const double d212c = dot3(v21[0], v21[1], v21[2], v2c[0], v2c[1], v2c[2]);
      const double d322c = dot3(v32[0], v32[1], v32[2], v2c[0], v2c[1], v2c[2]);
      const double d1c1c = dot3(v1c[0], v1c[1], v1c[2], v1c[0], v1c[1], v1c[2]);
      const double d1c31 = dot3(v1c[0], v1c[1], v1c[2], v31[0], v31[1], v31[2]);
      const double d2c2c = dot3(v2c[0], v2c[1], v2c[2], v2c[0], v2c[1], v2c[2]);
      const double d2c1c = dot3(v2c[0], v2c[1], v2c[2], v1c[0], v1c[1], v1c[2]);
      const double d3c31 = dot3(v3c[0], v3c[1], v3c[2], v31[0], v31[1], v31[2]);
      const double d3c32 = dot3(v3c[0], v3c[1], v3c[2], v32[0], v32[1], v32[2]);
      const double d3c3c = dot3(v3c[0], v3c[1], v3c[2], v3c[0], v3c[1], v3c[2]);
      // j-independent terms of the hy/hxy/hx denominators (each is recomputed identically on every
      // quadrature point in the reference, so evaluating it once gives the same double)
      const double p211 = d211c * d211c;
      const double p1121 = d1c1c * d2121;
      const double p3131sq = d1c31 * d1c31;
      const double p1131 = d1c1c * d3131;
      double t0 = 0.0, s0 = 0.0, sx = 0.0, sy = 0.0, sxy = 0.0, syy = 0.0, sxx = 0.0;
#pragma unroll 3
      for (int j = 0; j < 21; ++j) {
        const double y = c_gy[j], w = c_gw[j];
        const double y2 = 2.0 * y, yy = y * y;
        const double q1 = sqrt(d1c1c + y2 * d1c31 + yy * d3131);
        const double q2 = sqrt(d2c2c + y2 * d322c + yy * d3232);
        // h (triangleint.f:198-206): the denominator's root is d1c1c + (2 d1c31) y + (d3131 y) y
        const double hv = log((d212c + d2132 * y + s21 * q2) /
                              (d211c + d2131 * y + s21 * sqrt(d1c1c + 2 * d1c31 * y + d3131 * y * y))) /
                          s21;
        // hy (:222-234)
        const double hya = (d211c + y * d2131) / q1;
        const double hyb = (y * d2132 + d212c) / q2;
        const double hyc = (p211 - p1121 - y2 * d1c31 * d2121 + y2 * d211c * d2131 + yy * d2131 * d2131 -
                            yy * d2121 * d3131);
        const double hyv = (hya - hyb) / hyc;
        // hxy (:236-247)
        const double hxyb = (y * d211c - d2c1c - y2 * d1c31 - y * d2131 - yy * d3231) / q2;
        const double hxyc =
            (-p211 + p1121 + y2 * d1c31 * d2121 - y2 * d211c * d2131 - yy * (d2131 * d2131) + yy * d2121 * d3131);
        const double hxyv = (q1 + hxyb) / hxyc;
        // hx (:208-220)
        const double hxa = (-d1c31 - y * d2131) / sqrt(d1c1c + y2 * d211c + yy * d2121);
        const double hxb = (-(y * d3231) + d3c31) / sqrt(yy * d3232 - y2 * d3c32 + d3c3c);
        const double hxc = (-p3131sq - y2 * d1c31 * d2131 - yy * d2131 * d2131 + p1131 + y2 * d211c * d3131 +
                            yy * d2121 * d3131);
        const double hxv = (hxa + hxb) / hxc;
        // :122-130
        const double wy = w * y, wyy = wy * y;
        t0 = t0 + w * hv;
        s0 = s0 + w * hyv;
        sx = sx + w * hxyv;
        sy = sy + wy * hyv;
        sxy = sxy + wy * hxyv;
        syy = syy + wyy * hyv;
        sxx = sxx + wyy * hxv;
      }
      t0 = 0.5 * t0;
      s0 = 0.5 * s0;
      sx = 0.5 * sx;
      sy = 0.5 * sy;
      sxy = 0.5 * sxy;
      syy = 0.5 * syy;
      sxx = 0.5 * sxx;
      // tensor (:149-177) and G (:180-188)
      double tt[6];
      int q = 0;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b)
          tt[q++] = v1c[a] * v1c[b] * s0 + (v1c[a] * v21[b] + v21[a] * v1c[b]) * sx +
                    (v31[a] * v1c[b] + v1c[a] * v31[b]) * sy + (v21[a] * v31[b] + v31[a] * v21[b]) * sxy +
                    v21[a] * v21[b] * sxx + v31[a] * v31[b] * syy;
      // tt: t11 t12 t13 t22 t23 t33
      const double ar2 = 2.0 * D[7];
      const double g11 = ar2 * (t0 + cg * tt[0]);
      const double g21 = ar2 * tt[1] * cg;
      const double g22 = ar2 * (t0 + cg * tt[3]);
      const double g31 = ar2 * tt[2] * cg;
      const double g32 = ar2 * tt[4] * cg;
      const double g33 = ar2 * (t0 + cg * tt[5]);
      blk[0] = g11; blk[1] = g21; blk[2] = g31;
      blk[3] = g21; blk[4] = g22; blk[5] = g32;
      blk[6] = g31; blk[7] = g32; blk[8] = g33;
    }
    const size_t col0 = 3 * (size_t)(n2 - c0);
    if (defl.ndef > 0) {
      const int k = s_comp[si];
      if (k == comp1) {
        const double gk = defl.gdef[k - 1];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const double gdj = gk * defl.xmu[3 * (size_t)n2 + b];
#pragma unroll
          for (int a = 0; a < 3; ++a) blk[3 * a + b] = blk[3 * a + b] + gdj * xmu_i[a];
        }
      }
    }
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double* col = out + (col0 + b) * (size_t)ld + row0;
#pragma unroll
      for (int a = 0; a < 3; ++a) col[a] = blk[3 * a + b];
    }
    if (out32) {
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float* col = out32 + (col0 + b) * (size_t)ld32 + row0;
#pragma unroll
        for (int a = 0; a < 3; ++a) col[a] = __double2float_rn(blk[3 * a + b]);
      }
    }
  }
}

__global__ void __launch_bounds__(kTgtTile, BGPU_ASM_MIN_BLOCKS)
    k_assemble(const double* __restrict__ geo, const double* __restrict__ xc, const double* __restrict__ self9,
               double cg, int r0, int r1, int c0, int c1, double* __restrict__ out, long ld, DevDeflation defl,
               float* __restrict__ out32, long ld32) {
  assemble_tile(blockIdx.x, blockIdx.y, geo, xc, self9, cg, r0, r1, c0, c1, out, ld, defl, out32, ld32);
}

// Every mesh of a series in one launch: block b belongs to the mesh whose tile range holds it.
__global__ void __launch_bounds__(kTgtTile, BGPU_ASM_MIN_BLOCKS) k_assemble_series(const __grid_constant__ SeriesAssembly sa) {
  const int b = blockIdx.x;
  int i = 0;
  while (i + 1 < sa.count && b >= sa.tile0[i + 1]) ++i;
  const int local = b - sa.tile0[i];
  const int tx = (sa.mesh[i].n + kTgtTile - 1) / kTgtTile;
  const DevMesh& m = sa.mesh[i];
  assemble_tile(local % tx, local / tx, m.geo, m.xc, m.self9, m.cg, 0, m.n, 0, m.n, sa.out[i], sa.ld[i], sa.defl[i],
                nullptr, 0);
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
