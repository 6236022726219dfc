// Adjoint of BEST's assembly: gradients of results with respect to the triangle corners.
//
// For a result J(F) of the solutions F = GR^-1 B, the adjoint method gives
//     dJ = sum_c lambda_c . (dB_c - dGR F_c),   lambda_c = GR^-T dJ/dF_c
// (the transposed solve reuses the FP64 LU).  dGR is never stored: these kernels recompute GR's
// entries and contract their derivatives with the weights W_pq = -sum_c lambda_c(p) F_c(q)^T on the
// fly.  No counterpart in the reference, which has no derivatives.
//
//   k_pair_adjoint  the off-diagonal blocks (best/triangleint.f:1-247): a hand-written reverse sweep
//                   of the 21-point quadrature per (target, source) pair; one thread per source
//                   triangle (its own geometry in registers, its gradient accumulated in registers),
//                   targets staged in shared memory 16 at a time, the target-side gradient reduced
//                   across the block with warp shuffles; up to 3 results at once (K)
//   k_tri_adjoint   the O(N) per-triangle geometry — self block (best/tgetgr.f:33-147), incenter,
//                   area, unit normal — differentiated in forward mode (9 tangent directions)
//   reductions      fixed-order sums of the per-block partials (results do not depend on scheduling)
#include <cuda_runtime.h>

#include <algorithm>

#include "bgpu_internal.h"
#include "dual.cuh"

namespace bgpu {
namespace {

constexpr double kPi = 3.1415926535897932385;  // best/tgetgr.f:17
constexpr int kSrcBlock = 128;                  // sources per block (threads)
constexpr int kTgtTile = 16;                    // targets staged per step
constexpr int kTgtChunkMax = 256;               // targets per block at most (grid.y splits the rest)
constexpr int kMaxCols = 17;                    // adjoint columns (6 + 6 + 5)

// 21-point Gauss-Legendre rule on [0,1] (best/triangleint.f:66-108), as in the assembly
__constant__ double c_ay[21] = {
    3.1239146898052499e-3, 1.6386580716846853e-2, 3.9950332924799586e-2, 7.3318317708341358e-2,
    0.1157800182621610,    0.1664305979012938,    0.2241905820563901,    0.2878289398962806,
    0.3559893415987995,    0.4272190729195525,    0.5,                   0.5727809270804476,
    0.6440106584012005,    0.7121710601037194,    0.7758094179436099,    0.8335694020987062,
    0.8842199817378390,    0.9266816822916586,    0.9600496670752004,    0.9836134192831532,
    0.9968760853101948};
__constant__ double c_aw[21] = {
    1.601722825777433e-2, 3.695378977085249e-2, 5.713442542685720e-2, 7.610011362837930e-2,
    9.344442345603390e-2, 0.1087972991671484,   0.1218314160537285,   0.1322689386333375,
    0.1398873947910731,   0.1445244039899701,   0.1460811336496904,   0.1445244039899701,
    0.1398873947910731,   0.1322689386333375,   0.1218314160537285,   0.1087972991671484,
    9.344442345603390e-2, 7.610011362837930e-2, 5.713442542685720e-2, 3.695378977085249e-2,
    1.601722825777433e-2};

__device__ __forceinline__ double dot3v(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// sum_ab M_ab u_a v_b for a symmetric M given as (00 11 22 01 02 12)
__device__ __forceinline__ double quad(const double* M, const double* u, const double* v) {
  return M[0] * u[0] * v[0] + M[1] * u[1] * v[1] + M[2] * u[2] * v[2] + M[3] * (u[0] * v[1] + u[1] * v[0]) +
         M[4] * (u[0] * v[2] + u[2] * v[0]) + M[5] * (u[1] * v[2] + u[2] * v[1]);
}
// out += M v
__device__ __forceinline__ void symv_add(const double* M, const double* v, double s, double* out) {
  out[0] += s * (M[0] * v[0] + M[3] * v[1] + M[4] * v[2]);
  out[1] += s * (M[3] * v[0] + M[1] * v[1] + M[5] * v[2]);
  out[2] += s * (M[4] * v[0] + M[5] * v[1] + M[2] * v[2]);
}

// The source triangle's target-independent data
struct SrcGeo {
  double P[9];
  double v21[3], v31[3], v32[3];
  double d2121, d2131, d2132, d3131, d3232, d3231, s21, area;
};

// Reverse sweep of one pair integral: G (3x3, triangleint.f:180-188) of source S seen from target X,
// contracted with W[k] (row = target component, column = source component).  Adds to qbar[k]
// (dP1, dP2, dP3, darea) and sets xbar[k] (dX).
template <int K>
__device__ void pair_reverse(const SrcGeo& S, double cg, const double* X, const double (&W)[K][9],
                             double (&xbar)[K][3], double (&qbar)[K][10]) {
  double v1c[3], v2c[3], v3c[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v1c[c] = S.P[c] - X[c];
    v2c[c] = S.P[3 + c] - X[c];
    v3c[c] = S.P[6 + c] - X[c];
  }
  const double d2121 = S.d2121, d2131 = S.d2131, d2132 = S.d2132, d3131 = S.d3131, d3232 = S.d3232, d3231 = S.d3231;
  const double s21 = S.s21, is21 = 1.0 / s21;
  const double d211c = dot3v(S.v21, v1c), d212c = dot3v(S.v21, v2c), d322c = dot3v(S.v32, v2c);
  const double d1c1c = dot3v(v1c, v1c), d1c31 = dot3v(v1c, S.v31), d2c2c = dot3v(v2c, v2c), d2c1c = dot3v(v2c, v1c);
  const double d3c31 = dot3v(v3c, S.v31), d3c32 = dot3v(v3c, S.v32), d3c3c = dot3v(v3c, v3c);
  const double p211 = d211c * d211c, p1121 = d1c1c * d2121, p3131sq = d1c31 * d1c31, p1131 = d1c1c * d3131;
  // symmetric weights, and the cotangents of the seven quadrature sums (before their factor 1/2)
  double Ws[K][6], trW[K], R0[K], Rs0[K], Rsx[K], Rsy[K], Rsxy[K], Rsxx[K], Rsyy[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    Ws[k][0] = W[k][0];
    Ws[k][1] = W[k][4];
    Ws[k][2] = W[k][8];
    Ws[k][3] = 0.5 * (W[k][1] + W[k][3]);
    Ws[k][4] = 0.5 * (W[k][2] + W[k][6]);
    Ws[k][5] = 0.5 * (W[k][5] + W[k][7]);
    trW[k] = Ws[k][0] + Ws[k][1] + Ws[k][2];
    const double a2 = 2.0 * S.area, tcg = a2 * cg;  // G = 2 area (t0 I + cg tt)
    R0[k] = 0.5 * a2 * trW[k];
    Rs0[k] = 0.5 * tcg * quad(Ws[k], v1c, v1c);
    Rsx[k] = tcg * quad(Ws[k], v1c, S.v21);
    Rsy[k] = tcg * quad(Ws[k], v1c, S.v31);
    Rsxy[k] = tcg * quad(Ws[k], S.v21, S.v31);
    Rsxx[k] = 0.5 * tcg * quad(Ws[k], S.v21, S.v21);
    Rsyy[k] = 0.5 * tcg * quad(Ws[k], S.v31, S.v31);
  }
  double g2121[K], g2131[K], g2132[K], g3131[K], g3232[K], g3231[K], gs21[K], g211c[K], g212c[K], g322c[K],
      g1c1c[K], g1c31[K], g2c2c[K], g2c1c[K], g3c31[K], g3c32[K], g3c3c[K];
#pragma unroll
  for (int k = 0; k < K; ++k)
    g2121[k] = g2131[k] = g2132[k] = g3131[k] = g3232[k] = g3231[k] = gs21[k] = g211c[k] = g212c[k] = g322c[k] =
        g1c1c[k] = g1c31[k] = g2c2c[k] = g2c1c[k] = g3c31[k] = g3c32[k] = g3c3c[k] = 0.0;
  double t0 = 0.0, s0 = 0.0, sx = 0.0, sy = 0.0, sxy = 0.0, syy = 0.0, sxx = 0.0;
#pragma unroll 1
  for (int j = 0; j < 21; ++j) {
    const double y = c_ay[j], w = c_aw[j];
    const double y2 = 2.0 * y, yy = y * y, wy = w * y, wyy = wy * y;
    const double q1 = sqrt(d1c1c + y2 * d1c31 + yy * d3131), iq1 = 1.0 / q1;
    const double q2 = sqrt(d2c2c + y2 * d322c + yy * d3232), iq2 = 1.0 / q2;
    const double Nn = d212c + d2132 * y + s21 * q2, Dd = d211c + d2131 * y + s21 * q1;
    const double iN = 1.0 / Nn, iD = 1.0 / Dd;
    const double hv = log(Nn * iD) * is21;
    const double hya = (d211c + y * d2131) * iq1, hyb = (y * d2132 + d212c) * iq2;
    const double hyc = p211 - p1121 - y2 * d1c31 * d2121 + y2 * d211c * d2131 + yy * d2131 * d2131 - yy * d2121 * d3131;
    const double ihyc = 1.0 / hyc;
    const double hyv = (hya - hyb) * ihyc;
    const double hxyb = (y * d211c - d2c1c - y2 * d1c31 - y * d2131 - yy * d3231) * iq2;
    const double hxyv = -(q1 + hxyb) * ihyc;  // the denominator of hxy is -hyc
    const double r1 = sqrt(d1c1c + y2 * d211c + yy * d2121), ir1 = 1.0 / r1;
    const double r2 = sqrt(yy * d3232 - y2 * d3c32 + d3c3c), ir2 = 1.0 / r2;
    const double hxa = (-d1c31 - y * d2131) * ir1, hxb = (-y * d3231 + d3c31) * ir2;
    const double hxc = -p3131sq - y2 * d1c31 * d2131 - yy * d2131 * d2131 + p1131 + y2 * d211c * d3131 + yy * d2121 * d3131;
    const double ihxc = 1.0 / hxc;
    const double hxv = (hxa + hxb) * ihxc;
    t0 += w * hv;
    s0 += w * hyv;
    sx += w * hxyv;
    sy += wy * hyv;
    sxy += wy * hxyv;
    syy += wyy * hyv;
    sxx += wyy * hxv;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double bv = w * R0[k], byv = w * Rs0[k] + wy * Rsy[k] + wyy * Rsyy[k], bxyv = w * Rsx[k] + wy * Rsxy[k],
                   bxv = wyy * Rsxx[k];
      double gq1 = 0.0, gq2 = 0.0;
      // h = log(Nn / Dd) / s21
      const double c1 = bv * is21 * iN, c2 = -bv * is21 * iD;
      g212c[k] += c1;
      g2132[k] += c1 * y;
      gq2 += c1 * s21;
      gs21[k] += c1 * q2 + c2 * q1 - bv * hv * is21;
      g211c[k] += c2;
      g2131[k] += c2 * y;
      gq1 += c2 * s21;
      // hy = (hya - hyb) / hyc
      const double gya = byv * ihyc, gyb = -byv * ihyc;
      double gyc = -byv * hyv * ihyc;
      // hxy = (q1 + hxyb) / (-hyc)
      gq1 += -bxyv * ihyc;
      const double gxyb = -bxyv * ihyc;
      gyc += -bxyv * hxyv * ihyc;
      // hya, hyb
      g211c[k] += gya * iq1;
      g2131[k] += gya * y * iq1;
      gq1 += -gya * hya * iq1;
      g2132[k] += gyb * y * iq2;
      g212c[k] += gyb * iq2;
      gq2 += -gyb * hyb * iq2;
      // hxyb
      const double gnum = gxyb * iq2;
      gq2 += -gxyb * hxyb * iq2;
      g211c[k] += gnum * y;
      g2c1c[k] -= gnum;
      g1c31[k] -= gnum * y2;
      g2131[k] -= gnum * y;
      g3231[k] -= gnum * yy;
      // hyc
      g211c[k] += gyc * (2.0 * d211c + y2 * d2131);
      g1c1c[k] -= gyc * d2121;
      g2121[k] += gyc * (-d1c1c - y2 * d1c31 - yy * d3131);
      g1c31[k] -= gyc * y2 * d2121;
      g2131[k] += gyc * (y2 * d211c + 2.0 * yy * d2131);
      g3131[k] -= gyc * yy * d2121;
      // hx = (hxa + hxb) / hxc
      const double gx = bxv * ihxc, gxc = -bxv * hxv * ihxc;
      g1c31[k] -= gx * ir1;
      g2131[k] -= gx * y * ir1;
      const double gr1 = -gx * hxa * ir1;
      g1c1c[k] += gr1 * 0.5 * ir1;
      g211c[k] += gr1 * y * ir1;
      g2121[k] += gr1 * 0.5 * yy * ir1;
      g3231[k] -= gx * y * ir2;
      g3c31[k] += gx * ir2;
      const double gr2 = -gx * hxb * ir2;
      g3232[k] += gr2 * 0.5 * yy * ir2;
      g3c32[k] -= gr2 * y * ir2;
      g3c3c[k] += gr2 * 0.5 * ir2;
      g1c31[k] += gxc * (-2.0 * d1c31 - y2 * d2131);
      g2131[k] += gxc * (-y2 * d1c31 - 2.0 * yy * d2131);
      g1c1c[k] += gxc * d3131;
      g3131[k] += gxc * (d1c1c + y2 * d211c + yy * d2121);
      g211c[k] += gxc * y2 * d3131;
      g2121[k] += gxc * yy * d3131;
      // the roots q1, q2
      g1c1c[k] += gq1 * 0.5 * iq1;
      g1c31[k] += gq1 * y * iq1;
      g3131[k] += gq1 * 0.5 * yy * iq1;
      g2c2c[k] += gq2 * 0.5 * iq2;
      g322c[k] += gq2 * y * iq2;
      g3232[k] += gq2 * 0.5 * yy * iq2;
    }
  }
  t0 *= 0.5;
  s0 *= 0.5;
  sx *= 0.5;
  sy *= 0.5;
  sxy *= 0.5;
  syy *= 0.5;
  sxx *= 0.5;
  const double* v21 = S.v21;
  const double* v31 = S.v31;
  const double* v32 = S.v32;
  // tt (00 11 22 01 02 12), triangleint.f:149-177
  double tt[6];
  {
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      const int a = ia[e], b = ib[e];
      tt[e] = v1c[a] * v1c[b] * s0 + (v1c[a] * v21[b] + v21[a] * v1c[b]) * sx + (v31[a] * v1c[b] + v1c[a] * v31[b]) * sy +
              (v21[a] * v31[b] + v31[a] * v21[b]) * sxy + v21[a] * v21[b] * sxx + v31[a] * v31[b] * syy;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    g2121[k] += gs21[k] * 0.5 * is21;
    double g1c[3] = {0, 0, 0}, g21[3] = {0, 0, 0}, g31[3] = {0, 0, 0}, g32[3] = {0, 0, 0}, g2c[3] = {0, 0, 0},
           g3c[3] = {0, 0, 0};
    // from tt (the tensor's explicit dependence on the vectors)
    const double tcg2 = 2.0 * 2.0 * S.area * cg;
    double u[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = v1c[c] * s0 + v21[c] * sx + v31[c] * sy;
    symv_add(Ws[k], u, tcg2, g1c);
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = v1c[c] * sx + v31[c] * sxy + v21[c] * sxx;
    symv_add(Ws[k], u, tcg2, g21);
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = v1c[c] * sy + v21[c] * sxy + v31[c] * syy;
    symv_add(Ws[k], u, tcg2, g31);
    // from the dot products
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      g21[c] += 2.0 * g2121[k] * v21[c] + g2131[k] * v31[c] + g2132[k] * v32[c] + g211c[k] * v1c[c] + g212c[k] * v2c[c];
      g31[c] += g2131[k] * v21[c] + 2.0 * g3131[k] * v31[c] + g3231[k] * v32[c] + g1c31[k] * v1c[c] + g3c31[k] * v3c[c];
      g32[c] += g2132[k] * v21[c] + 2.0 * g3232[k] * v32[c] + g3231[k] * v31[c] + g322c[k] * v2c[c] + g3c32[k] * v3c[c];
      g1c[c] += g211c[k] * v21[c] + 2.0 * g1c1c[k] * v1c[c] + g1c31[k] * v31[c] + g2c1c[k] * v2c[c];
      g2c[c] += g212c[k] * v21[c] + g322c[k] * v32[c] + 2.0 * g2c2c[k] * v2c[c] + g2c1c[k] * v1c[c];
      g3c[c] += g3c31[k] * v31[c] + g3c32[k] * v32[c] + 2.0 * g3c3c[k] * v3c[c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      qbar[k][c] += -g21[c] - g31[c] + g1c[c];
      qbar[k][3 + c] += g21[c] - g32[c] + g2c[c];
      qbar[k][6 + c] += g31[c] + g32[c] + g3c[c];
      xbar[k][c] = -(g1c[c] + g2c[c] + g3c[c]);
    }
    double wtt = 0.0;
#pragma unroll
    for (int e = 0; e < 6; ++e) wtt += (e < 3 ? 1.0 : 2.0) * Ws[k][e] * tt[e];
    qbar[k][9] += 2.0 * (t0 * trW[k] + cg * wtt);
  }
}

// lam, fs: [t][C][3] (the adjoint vectors and the solutions of each column at triangle t); the
// column's result index in col_out.  xbar_part: [gridDim.x][n][3K]; qbar_part: [gridDim.y][n][10K].
struct ColMap {
  int out[kMaxCols];
};

template <int K>
__global__ void __launch_bounds__(kSrcBlock) k_pair_adjoint(int n, const double* __restrict__ geo,
                                                            const double* __restrict__ xc, double cg,
                                                            const double* __restrict__ lam,
                                                            const double* __restrict__ fs, int C, ColMap cols,
                                                            int tgt_chunk, double* __restrict__ xbar_part,
                                                            double* __restrict__ qbar_part) {
  extern __shared__ double sm[];
  const int stride = 3 * C;
  double* s_f = sm;                                     // [128][3C]: this block's sources' solutions
  double* s_t = s_f + kSrcBlock * stride;               // [16][3 + 3C]: staged targets (X, lambda)
  double* s_red = s_t + kTgtTile * (3 + stride);        // [4 warps][16][3K]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = blockIdx.x * kSrcBlock + tid;
  const bool qlive = q < n;
  for (int i = tid; i < kSrcBlock * stride; i += kSrcBlock) {
    const int qq = blockIdx.x * kSrcBlock + i / stride;
    s_f[i] = qq < n ? fs[(size_t)qq * stride + i % stride] : 0.0;
  }
  SrcGeo S;
  if (qlive) {
    const double* g = geo + (size_t)q * kGeoStride;
#pragma unroll
    for (int i = 0; i < 9; ++i) S.P[i] = g[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      S.v21[c] = S.P[3 + c] - S.P[c];
      S.v31[c] = S.P[6 + c] - S.P[c];
      S.v32[c] = S.P[6 + c] - S.P[3 + c];
    }
    S.d2121 = dot3v(S.v21, S.v21);
    S.d2131 = dot3v(S.v21, S.v31);
    S.d2132 = dot3v(S.v21, S.v32);
    S.d3131 = dot3v(S.v31, S.v31);
    S.d3232 = dot3v(S.v32, S.v32);
    S.d3231 = dot3v(S.v32, S.v31);
    S.s21 = sqrt(S.d2121);
    S.area = g[9];
  }
  double qacc[K][10];
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int i = 0; i < 10; ++i) qacc[k][i] = 0.0;
  const int p_lo = blockIdx.y * tgt_chunk, p_hi = min(n, p_lo + tgt_chunk);
  for (int t0 = p_lo; t0 < p_hi; t0 += kTgtTile) {
    const int nt = min(kTgtTile, p_hi - t0);
    __syncthreads();
    for (int i = tid; i < nt * (3 + stride); i += kSrcBlock) {
      const int tt = i / (3 + stride), e = i % (3 + stride);
      const int p = t0 + tt;
      s_t[i] = e < 3 ? xc[(size_t)p * kXcStride + e] : lam[(size_t)p * stride + (e - 3)];
    }
    __syncthreads();
    for (int tt = 0; tt < nt; ++tt) {
      const int p = t0 + tt;
      double xb[K][3];
#pragma unroll
      for (int k = 0; k < K; ++k) xb[k][0] = xb[k][1] = xb[k][2] = 0.0;
      if (qlive && p != q) {
        const double* tp = s_t + tt * (3 + stride);
        double W[K][9];
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
          for (int e = 0; e < 9; ++e) W[k][e] = 0.0;
        const double* fq = s_f + tid * stride;
        for (int c = 0; c < C; ++c) {
          const double* lp = tp + 3 + 3 * c;
          const double* fc = fq + 3 * c;
#pragma unroll
          for (int k = 0; k < K; ++k)
            if (cols.out[c] == k)
#pragma unroll
              for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) W[k][3 * a + b] -= lp[a] * fc[b];
        }
        pair_reverse<K>(S, cg, tp, W, xb, qacc);
      }
      // the target's gradient: sum over this block's sources
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double v = xb[k][c];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) s_red[(warp * kTgtTile + tt) * 3 * K + 3 * k + c] = v;
        }
    }
    __syncthreads();
    for (int i = tid; i < nt * 3 * K; i += kSrcBlock) {
      const int tt = i / (3 * K), e = i % (3 * K);
      double v = 0.0;
      for (int w = 0; w < kSrcBlock / 32; ++w) v += s_red[(w * kTgtTile + tt) * 3 * K + e];
      xbar_part[((size_t)blockIdx.x * n + t0 + tt) * 3 * K + e] = v;
    }
  }
  if (qlive)
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int i = 0; i < 10; ++i) qbar_part[((size_t)blockIdx.y * n + q) * 10 * K + 10 * k + i] = qacc[k][i];
}

// out[i] = sum_{b < parts} part[b * len + i], in order
__global__ void k_sum_parts(const double* __restrict__ part, int parts, size_t len, double* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  double s = 0.0;
  for (int b = 0; b < parts; ++b) s += part[(size_t)b * len + i];
  out[i] = s;
}

// ---- per-triangle geometry, generic in the scalar type (double or Dual<N>) ---------------------
// best/tgetgr.f:36-145 (incenter, unit normal, exact self integrals rotated to the lab frame) and
// the triangle's area (best/best.f:286-291) from its corners p (p1, p2, p3).
template <class T>
__host__ __device__ T si_t(const T& x) {
  const T r = sqrt(1.0 - x * x);
  return 2.0 * (log((1.0 + r) / x) - r);
}
template <class T>
__host__ __device__ T csi_t(const T& x) {
  return 3.0 - 1.0 / x - 2.0 * x;
}

template <class T>
__host__ __device__ void tri_geometry(const T* p, double cor, double cg, T* x, T& area_raw, T* nrm, T* self9) {
  const double pi = kPi;
  const T v21x = p[3] - p[0], v21y = p[4] - p[1], v21z = p[5] - p[2];
  const T v31x = p[6] - p[0], v31y = p[7] - p[1], v31z = p[8] - p[2];
  const T v32x = p[6] - p[3], v32y = p[7] - p[4], v32z = p[8] - p[5];
  const T a = sqrt(v21x * v21x + v21y * v21y + v21z * v21z);
  const T b = sqrt(v31x * v31x + v31y * v31y + v31z * v31z);
  const T c = sqrt(v32x * v32x + v32y * v32y + v32z * v32z);
  const T cosC = (v21x * v31x + v21y * v31y + v21z * v31z) / a / b;
  const T tin = (a + b - c) / (2. * (1. + cosC));
  x[0] = p[0] + tin * (v21x / a + v31x / b);
  x[1] = p[1] + tin * (v21y / a + v31y / b);
  x[2] = p[2] + tin * (v21z / a + v31z / b);
  T nx = v31y * v21z - v31z * v21y;
  T ny = v31z * v21x - v31x * v21z;
  T nz = v31x * v21y - v31y * v21x;
  const T area2 = sqrt(nx * nx + ny * ny + nz * nz) / 2.;
  area_raw = area2;
  nx = .5 * nx / area2;
  ny = .5 * ny / area2;
  nz = .5 * nz / area2;
  nrm[0] = nx;
  nrm[1] = ny;
  nrm[2] = nz;
  const T cc = acos(cosC);
  const T r = tin * sin(cc);
  const T cosB = -(v21x * v32x + v21y * v32y + v21z * v32z) / a / c;
  const T bb = acos(cosB);
  const T aa = pi - bb - cc;
  const T hcos = 1. / (2. * cos(0.5 * cc));
  const T dc = (a + b - c) * hcos;
  const T db = sqrt(a * a + (b - c) * (b - c) - 2. * a * (b - c) * cosC) * hcos;
  const T da = sqrt(b * b + (a - c) * (a - c) - 2. * b * (a - c) * cosC) * hcos;
  const T ha = r / da, hb = r / db, hc = r / dc;
  const T dpa = (pi - aa) * (da - r) - 2.0 * (da * acos(ha) - r * log((1. + sqrt(1. - ha * ha)) / ha));
  const T dpb = (pi - bb) * (db - r) - 2.0 * (db * acos(hb) - r * log((1. + sqrt(1. - hb * hb)) / hb));
  const T dpc = (pi - cc) * (dc - r) - 2.0 * (dc * acos(hc) - r * log((1. + sqrt(1. - hc * hc)) / hc));
  const T sca = 0.5 * r * ((cos(2.0 * cc) + cos(2.0 * bb)) * si_t(ha) - (sin(2.0 * cc) + sin(2.0 * bb)) * csi_t(ha));
  const T scb = 0.5 * r * ((1. + cos(2.0 * bb)) * si_t(hb) + sin(2.0 * bb) * csi_t(hb));
  const T scc = 0.5 * r * ((1. + cos(2.0 * cc)) * si_t(hc) + sin(2.0 * cc) * csi_t(hc));
  const T cca = -(sin(bb - cc) * r * (cos(aa) * si_t(ha) + sin(aa) * csi_t(ha)));
  const T ccb = sin(bb) * r * (cos(bb) * si_t(hb) + sin(bb) * csi_t(hb));
  const T ccc = -(sin(cc) * r * (cos(cc) * si_t(hc) + sin(cc) * csi_t(hc)));
  T gl[3][3];
  gl[0][0] = cor * ((2.0 + cg) * pi * r + (1.0 + 0.5 * cg) * cg * (dpa + dpb + dpc) + cg * 0.25 * (sca + scb + scc));
  gl[0][1] = 0.5 * cor * (cca + ccb + ccc) * cg;
  gl[1][0] = gl[0][1];
  gl[1][1] = gl[0][0] - 0.5 * cor * cg * (sca + scb + scc);
  gl[2][2] = cor * (2.0 * pi * r + (dpa + dpb + dpc));
  gl[0][2] = gl[1][2] = gl[2][0] = gl[2][1] = T(0.0);
  T rr[3][3];
  rr[0][0] = v21x / a;
  rr[0][1] = v21y / a;
  rr[0][2] = v21z / a;
  rr[2][0] = nx;
  rr[2][1] = ny;
  rr[2][2] = nz;
  rr[1][0] = (ny * v21z - nz * v21y) / a;
  rr[1][1] = (nz * v21x - nx * v21z) / a;
  rr[1][2] = (nx * v21y - ny * v21x) / a;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T acc(0.0);
      for (int k = 0; k < 3; ++k) acc = acc + rr[k][i] * (gl[k][0] * rr[0][j] + gl[k][1] * rr[1][j] + gl[k][2] * rr[2][j]);
      self9[3 * i + j] = acc;
    }
}

// cot: [t][K][16] = cotangents of self9 (9), incenter (3), raw area (1), unit normal (3);
// vbar: [t][K][9] = their pull-back to the corners p1, p2, p3.
template <int K>
__global__ void __launch_bounds__(64) k_tri_adjoint(int n, const double* __restrict__ geo, double cor, double cg,
                                                    const double* __restrict__ cot, double* __restrict__ vbar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  using D = Dual<9>;
  D p[9], x[3], area, nrm[3], s9[9];
  for (int i = 0; i < 9; ++i) p[i] = D::var(geo[(size_t)t * kGeoStride + i], i);
  tri_geometry<D>(p, cor, cg, x, area, nrm, s9);
  for (int k = 0; k < K; ++k) {
    const double* ck = cot + ((size_t)t * K + k) * 16;
    double g[9];
    for (int i = 0; i < 9; ++i) {
      double v = 0.0;
      for (int e = 0; e < 9; ++e) v += ck[e] * s9[e].d[i];
      for (int c = 0; c < 3; ++c) v += ck[9 + c] * x[c].d[i];
      v += ck[12] * area.d[i];
      for (int c = 0; c < 3; ++c) v += ck[13 + c] * nrm[c].d[i];
      g[i] = v;
    }
    for (int i = 0; i < 9; ++i) vbar[((size_t)t * K + k) * 9 + i] = g[i];
  }
}

// targets per block: at most kTgtChunkMax, and few enough that the grid has two blocks per SM
int tgt_chunk(int n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int gx = (n + kSrcBlock - 1) / kSrcBlock;
  const int gy = std::max(1, (2 * sms + gx - 1) / gx);
  int chunk = (n + gy - 1) / gy;
  chunk = (chunk + kTgtTile - 1) / kTgtTile * kTgtTile;
  return std::max(kTgtTile, std::min(kTgtChunkMax, chunk));
}

template <int K>
cudaError_t run_pair(const DevMesh& m, const double* lam, const double* fs, int C, const int* col_out, double* xbar,
                     double* qbar, double* scratch, cudaStream_t s) {
  ColMap cols{};
  for (int c = 0; c < C; ++c) cols.out[c] = col_out[c];
  const int gx = (m.n + kSrcBlock - 1) / kSrcBlock, chunk = tgt_chunk(m.n), gy = (m.n + chunk - 1) / chunk;
  const size_t smem = (size_t)(kSrcBlock * 3 * C + kTgtTile * (3 + 3 * C) + 4 * kTgtTile * 3 * K) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(k_pair_adjoint<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  double* xpart = scratch;
  double* qpart = scratch + (size_t)gx * m.n * 3 * K;
  k_pair_adjoint<K><<<dim3(gx, gy), kSrcBlock, smem, s>>>(m.n, m.geo, m.xc, m.cg, lam, fs, C, cols, chunk, xpart,
                                                           qpart);
  BGPU_COUNT_LAUNCH();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const size_t lx = (size_t)m.n * 3 * K, lq = (size_t)m.n * 10 * K;
  k_sum_parts<<<(unsigned)((lx + 255) / 256), 256, 0, s>>>(xpart, gx, lx, xbar);
  BGPU_COUNT_LAUNCH();
  k_sum_parts<<<(unsigned)((lq + 255) / 256), 256, 0, s>>>(qpart, gy, lq, qbar);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace

size_t pair_adjoint_scratch_bytes(int n, int K) {
  const size_t gx = (n + kSrcBlock - 1) / kSrcBlock, chunk = tgt_chunk(n), gy = (n + chunk - 1) / chunk;
  return (gx * n * 3 * K + gy * n * 10 * K) * sizeof(double);
}

cudaError_t launch_pair_adjoint(const DevMesh& m, int K, const double* lam, const double* fs, int C,
                                const int* col_out, double* xbar, double* qbar, void* scratch, cudaStream_t s) {
  if (C < 1 || C > kMaxCols || K < 1 || K > 3) return cudaErrorInvalidValue;
  double* sc = static_cast<double*>(scratch);
  switch (K) {
    case 1: return run_pair<1>(m, lam, fs, C, col_out, xbar, qbar, sc, s);
    case 2: return run_pair<2>(m, lam, fs, C, col_out, xbar, qbar, sc, s);
    default: return run_pair<3>(m, lam, fs, C, col_out, xbar, qbar, sc, s);
  }
}

cudaError_t launch_tri_adjoint(const DevMesh& m, int K, const double* cot, double* vbar, cudaStream_t s) {
  if (K < 1 || K > 3) return cudaErrorInvalidValue;
  const double cor = sqrt(m.afac);
  const unsigned g = (unsigned)((m.n + 63) / 64);
  switch (K) {
    case 1: k_tri_adjoint<1><<<g, 64, 0, s>>>(m.n, m.geo, cor, m.cg, cot, vbar); break;
    case 2: k_tri_adjoint<2><<<g, 64, 0, s>>>(m.n, m.geo, cor, m.cg, cot, vbar); break;
    default: k_tri_adjoint<3><<<g, 64, 0, s>>>(m.n, m.geo, cor, m.cg, cot, vbar); break;
  }
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace bgpu
