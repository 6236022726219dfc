// The pair-integral tile of the GR assembly (best/triangleint.f:1-247, hmatrix/src/kernel.cpp:148-249;
// epilogue: the deflation term of best/best.f:406-425 and an optional FP32 copy), shared by the
// bit-exact kernel (assemble.cu, compiled with -fmad=false) and the mixed path's kernel
// (assemble_fast.cu): each file instantiates one variant.
#pragma once
#include <cuda_runtime.h>

#include "bgpu_internal.h"
#include "ddmath.cuh"

namespace bgpu {
namespace {

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

// Target-independent terms of source triangle gp (kGeoStride doubles: p1, p2, p3, ..., area at 9):
// P = p1, p2, p3; V = v21, v31, v32; D = d2121 d2131 d2132 d3131 d3232 d3231 s21 area 1/s21 (the
// last for Fast only).  triangleint.f:110-120 (kernel.cpp:160-172).
template <bool Fast>
__device__ __forceinline__ void source_terms(const double* __restrict__ gp, double* P, double* V, double* D) {
  double p[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) p[q] = gp[q];
#pragma unroll
  for (int q = 0; q < 9; ++q) P[q] = p[q];
  double v21[3], v31[3], v32[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v21[c] = p[3 + c] - p[c];
    v31[c] = p[6 + c] - p[c];
    v32[c] = p[6 + c] - p[3 + c];
    V[c] = v21[c];
    V[3 + c] = v31[c];
    V[6 + c] = v32[c];
  }
  const double d2121 = dot3(v21[0], v21[1], v21[2], v21[0], v21[1], v21[2]);
  D[0] = d2121;
  D[1] = dot3(v21[0], v21[1], v21[2], v31[0], v31[1], v31[2]);
  D[2] = dot3(v21[0], v21[1], v21[2], v32[0], v32[1], v32[2]);
  D[3] = dot3(v31[0], v31[1], v31[2], v31[0], v31[1], v31[2]);
  D[4] = dot3(v32[0], v32[1], v32[2], v32[0], v32[1], v32[2]);
  D[5] = dot3(v32[0], v32[1], v32[2], v31[0], v31[1], v31[2]);
  D[6] = sqrt(d2121);
  D[7] = gp[9];
  if constexpr (Fast) D[8] = 1.0 / D[6];
}

// The 3 x 3 block G(target, source) of one pair of distinct triangles (triangleint.f:110-188,
// kernel.cpp:148-249): P, V, D the source's terms (source_terms), xc the target's incenter;
// blk[3a + b] = G_ab.  Fast = false needs s_logtab (the shared copy of the log's table).
template <bool Fast>
__device__ __forceinline__ void pair_gr(const double* P, const double* V, const double* D, double xcx, double xcy,
                                        double xcz, double cg, const double* s_logtab, double* blk) {
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
  double t0 = 0.0, s0 = 0.0, sx = 0.0, sy = 0.0, sxy = 0.0, syy = 0.0, sxx = 0.0;
  if constexpr (!Fast) {
    // j-independent terms of the hy/hxy/hx denominators (each is recomputed identically on every
    // quadrature point in the reference, so evaluating it once gives the same double)
    const double p211 = d211c * d211c;
    const double p1121 = d1c1c * d2121;
    const double p3131sq = d1c31 * d1c31;
    const double p1131 = d1c1c * d3131;
#pragma unroll 3
    for (int j = 0; j < 21; ++j) {
      const double y = c_gy[j], w = c_gw[j];
      const double y2 = 2.0 * y, yy = y * y;
      const double q1 = sqrt(d1c1c + y2 * d1c31 + yy * d3131);
      const double q2 = sqrt(d2c2c + y2 * d322c + yy * d3232);
      // h (triangleint.f:198-206): the denominator's root is d1c1c + (2 d1c31) y + (d3131 y) y
      const double hv = dd::cr_log_tab((d212c + d2132 * y + s21 * q2) /
                                           (d211c + d2131 * y + s21 * sqrt(d1c1c + 2 * d1c31 * y + d3131 * y * y)),
                                       s_logtab) /
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
  } else {
    // 1/sqrt as rsqrt (q = a rsqrt(a)); the denominators of hy and hxy (exact negatives of each
    // other in triangleint.f) and of hx as quadratics in y with per-pair coefficients; one
    // reciprocal per quadrature point for all three quotients; 1/s21 once per source triangle
    const double inv_s21 = D[8];
    const double cy0 = d211c * d211c - d1c1c * d2121;
    const double cy1 = 2.0 * (d211c * d2131 - d1c31 * d2121);
    const double cy2 = d2131 * d2131 - d2121 * d3131;
    const double cx0 = d1c1c * d3131 - d1c31 * d1c31;
    const double cx1 = 2.0 * (d211c * d3131 - d1c31 * d2131);
#pragma unroll 3
    for (int j = 0; j < 21; ++j) {
      const double y = c_gy[j], w = c_gw[j];
      const double a1 = d1c1c + y * (2.0 * d1c31 + y * d3131);
      const double a2 = d2c2c + y * (2.0 * d322c + y * d3232);
      const double a3 = d1c1c + y * (2.0 * d211c + y * d2121);
      const double a4 = d3c3c + y * (y * d3232 - 2.0 * d3c32);
      const double r1 = rsqrt(a1), r2 = rsqrt(a2);
      const double q1 = a1 * r1, q2 = a2 * r2;
      // the three quotients (log argument, hy/hxy, hx) from one reciprocal of the product of
      // their denominators (that product scales as the 10th power of the mesh's size: meshes
      // whose extent lies outside [1e-20, 1e20] are assembled by the exact kernel instead,
      // DevMesh::fast_ok)
      const double den = d211c + d2131 * y + s21 * q1;
      const double dy = cy0 + y * (cy1 + y * cy2), dx = cx0 + y * (cx1 - y * cy2);
      const double dyx = dy * dx;
      const double r = 1.0 / (dyx * den);
      const double ry = dx * den * r, rx = dy * den * r, rden = dyx * r;
      const double hv = log((d212c + d2132 * y + s21 * q2) * rden) * inv_s21;
      const double hyv = ((d211c + y * d2131) * r1 - (y * d2132 + d212c) * r2) * ry;
      const double hxyv = -(q1 + (y * d211c - d2c1c - 2.0 * y * d1c31 - y * d2131 - y * y * d3231) * r2) * ry;
      const double hxv = ((-d1c31 - y * d2131) * rsqrt(a3) + (d3c31 - y * d3231) * rsqrt(a4)) * rx;
      const double wy = w * y, wyy = wy * y;
      t0 = t0 + w * hv;
      s0 = s0 + w * hyv;
      sx = sx + w * hxyv;
      sy = sy + wy * hyv;
      sxy = sxy + wy * hxyv;
      syy = syy + wyy * hyv;
      sxx = sxx + wyy * hxv;
    }
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

// One tile: targets [r0 + 128 bx, +128) x sources [c0 + 16 by, +16) of one mesh.  Fast = false:
// triangleint.f's operations in its order with a correctly rounded log (bit for bit TGETGR's
// arithmetic with correctly rounded functions; the including file is compiled with -fmad=false);
// s_logtab: the block's shared copy of the log's reduction table, filled here.  Fast = true: the same
// integrals with fewer FP64 operations and the hardware log, for the mixed path (s_logtab unused).
template <bool Fast>
__device__ __forceinline__ void assemble_tile(int bx, int by, const double* __restrict__ geo,
                                              const double* __restrict__ xc, const double* __restrict__ self9,
                                              double cg, int r0, int r1, int c0, int c1, double* __restrict__ out,
                                              long ld, const DevDeflation& defl, float* __restrict__ out32, long ld32,
                                              double* s_logtab) {
  __shared__ double s_p[kSrcTile][9];     // p1, p2, p3
  __shared__ double s_v[kSrcTile][9];     // v21, v31, v32
  __shared__ double s_d[kSrcTile][9];     // d2121 d2131 d2132 d3131 d3232 d3231 s21 area 1/s21
  __shared__ int s_comp[kSrcTile];

  const int sbase = c0 + by * kSrcTile;
  const int ns = min(kSrcTile, c1 - sbase);
  if (threadIdx.x < ns) {
    const int t = sbase + threadIdx.x;
    source_terms<Fast>(geo + (size_t)t * kGeoStride, s_p[threadIdx.x], s_v[threadIdx.x], s_d[threadIdx.x]);
    s_comp[threadIdx.x] = (defl.ndef > 1) ? defl.comp[t] : 1;
  }
  if constexpr (!Fast) {
    for (int q = threadIdx.x; q < 3 * dd::kLogTabN; q += blockDim.x) s_logtab[q] = dd::kLogTab[q];
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
      pair_gr<Fast>(s_p[si], s_v[si], s_d[si], xcx, xcy, xcz, cg, s_logtab, blk);
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

}  // namespace
}  // namespace bgpu
