// The hierarchical-matrix path for meshes beyond the dense paths' reach (N above ~40,000 on one B200): GR held as dense
// near-field blocks and low-rank far-field blocks, solved by FP64 GMRES.
//
// Compiled with -fmad=false: every entry this path evaluates (the dense blocks in full, the rows
// and columns the cross approximation samples) comes from assemble_tile.cuh's exact pair kernel and
// equals the entry bhm_entries returns bit for bit.
//
// Reference: hmatrix/src/cluster.cpp (cluster tree, admissibility), hmatrix/src/hmatrix.cpp:26-60
// (block structure), :71-276 (ACA fill), hmatrix/src/gmres.cpp:26-180 (restarted GMRES over several
// right-hand sides), hmatrix/src/api.cpp:582-771 (build, deflation as a low-rank term, solve).
// Design for the B200:
//   * the triangles are permuted into tree order once, so every block is a contiguous range of rows
//     and columns and the pair tiles of the dense assembly fill any block unchanged;
//   * near blocks: one launch over the tiles of all dense blocks;
//   * far blocks: cross approximation with 3 x 3 pivots, batched over every block at once: each step
//     is four launches (the pivot row triangle's 3 rows, their residual and the next pivot column,
//     that triangle's 3 columns, their residual, the 3 x 3 pivot's inverse and the stopping test);
//   * product: the far blocks' V^T x (a warp per rank-one term), then one CTA per leaf row cluster
//     sums its dense blocks, its share of every low-rank block above it and the deflation term, in a
//     fixed order (no atomics: the product is deterministic);
//   * preconditioner: block Jacobi on the leaf diagonal blocks (with the deflation term), inverted
//     by Gauss-Jordan with partial pivoting, one CTA per leaf;
//   * GMRES(30), right-preconditioned, all right-hand sides in lockstep, classical Gram-Schmidt
//     with one reorthogonalisation, true residual at every restart.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "assemble_tile.cuh"
#include "bgpu_internal.h"
#include "hmatrix.h"

namespace bgpu {

// ---------------------------------------------------------------------------------------------
// Host: cluster tree and block partition
// ---------------------------------------------------------------------------------------------

namespace {

void hsplit(HPlan& p, const double* geo, const double* xc, int id) {
  HPlan::Cluster c = p.cl[id];
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = 1e300;
    c.hi[d] = -1e300;
  }
  for (int k = c.beg; k < c.beg + c.cnt; ++k) {
    const double* g = geo + (size_t)p.perm[k] * kGeoStride;
    for (int v = 0; v < 3; ++v)
      for (int d = 0; d < 3; ++d) {
        c.lo[d] = std::min(c.lo[d], g[3 * v + d]);
        c.hi[d] = std::max(c.hi[d], g[3 * v + d]);
      }
  }
  if (c.level == p.depth) {
    c.son0 = -1;
    p.cl[id] = c;
    p.leaves.push_back(id);
    return;
  }
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int k = c.beg; k < c.beg + c.cnt; ++k) {
    const double* x = xc + (size_t)p.perm[k] * kXcStride;
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], x[d]);
      hi[d] = std::max(hi[d], x[d]);
    }
  }
  int axis = 0;
  for (int d = 1; d < 3; ++d)
    if (hi[d] - lo[d] > hi[axis] - lo[axis]) axis = d;
  // the half smallest by (coordinate, triangle): the reference's nth_element selects the same set;
  // a full sort also fixes the order inside each half
  int* b = p.perm.data() + c.beg;
  std::sort(b, b + c.cnt, [&](int u, int v) {
    const double xu = xc[(size_t)u * kXcStride + axis], xv = xc[(size_t)v * kXcStride + axis];
    return xu < xv || (xu == xv && u < v);
  });
  const int half = c.cnt / 2;
  HPlan::Cluster s0, s1;
  s0.beg = c.beg;
  s0.cnt = half;
  s1.beg = c.beg + half;
  s1.cnt = c.cnt - half;
  s0.level = s1.level = c.level + 1;
  c.son0 = (int)p.cl.size();
  p.cl[id] = c;
  p.cl.push_back(s0);
  p.cl.push_back(s1);
  hsplit(p, geo, xc, c.son0);
  hsplit(p, geo, xc, c.son0 + 1);
}

double hdiam(const HPlan::Cluster& t) {
  double s = 0;
  for (int d = 0; d < 3; ++d) s += (t.hi[d] - t.lo[d]) * (t.hi[d] - t.lo[d]);
  return std::sqrt(s);
}

double hdist(const HPlan::Cluster& t, const HPlan::Cluster& u) {
  double s = 0;
  for (int d = 0; d < 3; ++d) {
    const double gap = std::max(0.0, std::max(t.lo[d] - u.hi[d], u.lo[d] - t.hi[d]));
    s += gap * gap;
  }
  return std::sqrt(s);
}

}  // namespace

HPlan hplan_build(int n, const double* geo, const double* xc, int leaf, double eta, int kmax) {
  HPlan p;
  p.n = n;
  if (n < 1 || leaf < 1) throw std::runtime_error("H-matrix plan: no triangles or leaf size < 1");
  p.perm.resize(n);
  std::iota(p.perm.begin(), p.perm.end(), 0);
  while ((((long)n + (1L << p.depth) - 1) >> p.depth) > leaf) ++p.depth;
  p.cl.reserve((size_t)2 << p.depth);
  HPlan::Cluster root;
  root.cnt = n;
  p.cl.push_back(root);
  hsplit(p, geo, xc, 0);
  // block tree from (root, root), leaves collected depth first (sons in order 00, 01, 10, 11)
  std::vector<std::pair<int, int>> stack{{0, 0}};
  while (!stack.empty()) {
    const auto [t, s] = stack.back();
    stack.pop_back();
    const HPlan::Cluster &ct = p.cl[t], &cs = p.cl[s];
    if (t != s && std::min(hdiam(ct), hdiam(cs)) <= eta * hdist(ct, cs)) {
      HPlan::Block b;
      b.t = t;
      b.s = s;
      b.admissible = true;
      // a cross approximation of kmax terms holds 3 (nr + nc) kmax entries
      b.lowrank = 9.0 * ct.cnt * cs.cnt > 3.0 * (ct.cnt + cs.cnt) * kmax;
      p.blocks.push_back(b);
    } else if (ct.son0 < 0 || cs.son0 < 0) {
      HPlan::Block b;
      b.t = t;
      b.s = s;
      p.blocks.push_back(b);
    } else {
      for (int i = 1; i >= 0; --i)
        for (int j = 1; j >= 0; --j) stack.push_back({ct.son0 + i, cs.son0 + j});
    }
  }
  return p;
}

// ---------------------------------------------------------------------------------------------
// Device
// ---------------------------------------------------------------------------------------------

namespace {

constexpr int kHQ = 16;          // right-hand sides per product
constexpr int kHMaxRank = 120;   // largest kmax
constexpr int kHMaxLeaf = 128;   // largest leaf (384 rows)
constexpr int kAcaThreads = 128;

struct HDense {
  int r0, nr, c0, nc;  // tree positions of the first target and source triangles, counts
  long long off;       // data at off, column-major, ld 3 nr
};
struct HLow {
  int r0, nr, c0, nc;
  long long uoff, voff;  // U: 3 nr x kcap (ld 3 nr), V: 3 nc x kcap (ld 3 nc)
  int kcap, toff;        // toff: the block's first rank-one term in the product's t array
};
struct HLeaf {
  int beg, cnt;          // tree positions
  int d0, d1, l0, l1;    // the leaf's dense and low-rank entries in the lists
  long long inv;         // offset of its diagonal block's inverse (3 cnt x 3 cnt)
  int diag;              // its diagonal dense block
  int pad;
};
struct HEntry {
  int blk;     // dense or low-rank block
  int rowoff;  // 3 (leaf.beg - block.r0)
};
struct AcaState {
  int rank, prow, pcol, active;
  int capped, pad0, pad1, pad2;
  double norm2;
};

__device__ __forceinline__ int find_tile(const int* __restrict__ tile0, int count, int b) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile0[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// gathered mesh in tree order
__global__ void k_tree_gather(int n, const int* __restrict__ perm, const double* __restrict__ geo,
                              const double* __restrict__ xc, const double* __restrict__ self9, double* __restrict__ geo_t,
                              double* __restrict__ xc_t, double* __restrict__ self9_t) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int t = perm[k];
  for (int q = 0; q < kGeoStride; ++q) geo_t[(size_t)k * kGeoStride + q] = geo[(size_t)t * kGeoStride + q];
  for (int q = 0; q < kXcStride; ++q) xc_t[(size_t)k * kXcStride + q] = xc[(size_t)t * kXcStride + q];
  for (int q = 0; q < 9; ++q) self9_t[(size_t)k * 9 + q] = self9[(size_t)t * 9 + q];
}

__global__ void k_defl_gather(int n, const int* __restrict__ perm, const double* __restrict__ xmu,
                              const int* __restrict__ comp, double* __restrict__ xmu_t, int* __restrict__ comp_t) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int t = perm[k];
  for (int a = 0; a < 3; ++a) xmu_t[3 * (size_t)k + a] = xmu[3 * (size_t)t + a];
  comp_t[k] = comp ? comp[t] : 1;
}

// Dense blocks: the exact pair tiles (assemble_tile<false>) into each block's storage.
__global__ void __launch_bounds__(kTgtTile, 4)
    k_fill_dense(const HDense* __restrict__ blk, const int* __restrict__ tile0, int nblk, const double* __restrict__ geo,
                 const double* __restrict__ xc, const double* __restrict__ self9, double cg, double* __restrict__ data) {
  __shared__ double s_logtab[3 * dd::kLogTabN];
  const int b = find_tile(tile0, nblk, blockIdx.x);
  const HDense B = blk[b];
  const int local = blockIdx.x - tile0[b];
  const int tx = (B.nr + kTgtTile - 1) / kTgtTile;
  DevDeflation none;
  assemble_tile<false>(local % tx, local / tx, geo, xc, self9, cg, B.r0, B.r0 + B.nr, B.c0, B.c0 + B.nc, data + B.off,
                       3L * B.nr, none, nullptr, 0, s_logtab);
}

__device__ __forceinline__ void pair_block(const double* __restrict__ geo, const double* __restrict__ xc,
                                           const double* __restrict__ self9, double cg, int ti, int sj,
                                           const double* s_logtab, double* blk) {
  if (ti == sj) {
#pragma unroll
    for (int q = 0; q < 9; ++q) blk[q] = self9[(size_t)ti * 9 + q];
    return;
  }
  double P[9], V[9], D[9];
  source_terms<false>(geo + (size_t)sj * kGeoStride, P, V, D);
  pair_gr<false>(P, V, D, xc[(size_t)ti * kXcStride], xc[(size_t)ti * kXcStride + 1], xc[(size_t)ti * kXcStride + 2],
                 cg, s_logtab, blk);
}

// ACA row step: V[:, k + a] = G(pivot row triangle's row a, all source columns) (thread per source).
__global__ void __launch_bounds__(kAcaThreads)
    k_aca_rows(const HLow* __restrict__ lb, const int* __restrict__ tile0, int nlb, const AcaState* __restrict__ st,
               const double* __restrict__ geo, const double* __restrict__ xc, const double* __restrict__ self9, double cg,
               double* __restrict__ Vp) {
  __shared__ double s_logtab[3 * dd::kLogTabN];
  const int b = find_tile(tile0, nlb, blockIdx.x);
  if (!st[b].active) return;
  for (int q = threadIdx.x; q < 3 * dd::kLogTabN; q += blockDim.x) s_logtab[q] = dd::kLogTab[q];
  __syncthreads();
  const HLow B = lb[b];
  const int j = (blockIdx.x - tile0[b]) * kAcaThreads + threadIdx.x;
  if (j >= B.nc) return;
  const int k = st[b].rank;
  double blk[9];
  pair_block(geo, xc, self9, cg, B.r0 + st[b].prow, B.c0 + j, s_logtab, blk);
  const long ldv = 3L * B.nc;
  double* V = Vp + B.voff;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) V[(size_t)(k + a) * ldv + 3 * j + c] = blk[3 * a + c];
}

// ACA column step: U[:, k + c] = G(all target rows, pivot column triangle's column c).
__global__ void __launch_bounds__(kAcaThreads)
    k_aca_cols(const HLow* __restrict__ lb, const int* __restrict__ tile0, int nlb, const AcaState* __restrict__ st,
               const double* __restrict__ geo, const double* __restrict__ xc, const double* __restrict__ self9, double cg,
               double* __restrict__ Up) {
  __shared__ double s_logtab[3 * dd::kLogTabN];
  const int b = find_tile(tile0, nlb, blockIdx.x);
  if (!st[b].active) return;
  for (int q = threadIdx.x; q < 3 * dd::kLogTabN; q += blockDim.x) s_logtab[q] = dd::kLogTab[q];
  __syncthreads();
  const HLow B = lb[b];
  const int i = (blockIdx.x - tile0[b]) * kAcaThreads + threadIdx.x;
  if (i >= B.nr) return;
  const int k = st[b].rank;
  double blk[9];
  pair_block(geo, xc, self9, cg, B.r0 + i, B.c0 + st[b].pcol, s_logtab, blk);
  const long ldu = 3L * B.nr;
  double* U = Up + B.uoff;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) U[(size_t)(k + c) * ldu + 3 * i + a] = blk[3 * a + c];
}

template <int NT>
__device__ __forceinline__ void block_argmax(double v, int idx, double* s_v, int* s_i, double* out_v, int* out_i) {
  // largest v, ties (and NaN-free equal values) to the smallest index
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, v, o);
    const int i2 = __shfl_down_sync(0xffffffffu, idx, o);
    if (v2 > v || (v2 == v && i2 < idx)) {
      v = v2;
      idx = i2;
    }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    s_v[w] = v;
    s_i[w] = idx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bv = s_v[0];
    int bi = s_i[0];
    for (int q = 1; q < NT / 32; ++q)
      if (s_v[q] > bv || (s_v[q] == bv && s_i[q] < bi)) {
        bv = s_v[q];
        bi = s_i[q];
      }
    *out_v = bv;
    *out_i = bi;
  }
  __syncthreads();
}

constexpr int kFixThreads = 256;

// Row residual: V[:, k..k+2] -= V[:, :k] U[3 prow + (0..2), :k]^T; the next pivot column (the source
// triangle whose 3 x 3 residual block is largest).  A zero residual row ends the block.
__global__ void __launch_bounds__(kFixThreads)
    k_aca_row_fix(const HLow* __restrict__ lb, AcaState* __restrict__ st, const double* __restrict__ Up,
                  double* __restrict__ Vp) {
  __shared__ double su[3][kHMaxRank];
  __shared__ double s_v[kFixThreads / 32];
  __shared__ int s_i[kFixThreads / 32];
  __shared__ double s_best;
  __shared__ int s_bi;
  const int b = blockIdx.x;
  if (!st[b].active) return;
  const HLow B = lb[b];
  const int k = st[b].rank, i = st[b].prow;
  const long ldu = 3L * B.nr, ldv = 3L * B.nc;
  const double* U = Up + B.uoff;
  double* V = Vp + B.voff;
  for (int q = threadIdx.x; q < 3 * k; q += blockDim.x) su[q % 3][q / 3] = U[(size_t)(q / 3) * ldu + 3 * i + q % 3];
  __syncthreads();
  double best = -1.0;
  int bi = 0x7fffffff;
  for (int s = threadIdx.x; s < B.nc; s += blockDim.x) {
    double nrm = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int row = 3 * s + c;
      double acc[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < k; ++q) {
        const double v = V[(size_t)q * ldv + row];
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] += su[a][q] * v;
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double r = V[(size_t)(k + a) * ldv + row] - acc[a];
        V[(size_t)(k + a) * ldv + row] = r;
        nrm += r * r;
      }
    }
    if (nrm > best) {
      best = nrm;
      bi = s;
    }
  }
  block_argmax<kFixThreads>(best, bi, s_v, s_i, &s_best, &s_bi);
  if (threadIdx.x == 0) {
    if (!(s_best > 0.0) || !isfinite(s_best)) st[b].active = 0;
    else st[b].pcol = s_bi;
  }
}

// Column residual, the pivot's inverse, the new terms U_new = C P^-1 (V_new = the residual rows),
// the Frobenius-norm update and the stopping test; the next pivot row.
__global__ void __launch_bounds__(kFixThreads)
    k_aca_col_fix(const HLow* __restrict__ lb, AcaState* __restrict__ st, double eps, double* __restrict__ Up,
                  const double* __restrict__ Vp) {
  __shared__ double sv[3][kHMaxRank];
  __shared__ double s_pinv[9];
  __shared__ int s_ok;
  __shared__ double s_red[kFixThreads / 32][24];
  __shared__ double s_cross[kHMaxRank];
  __shared__ double s_v[kFixThreads / 32];
  __shared__ int s_i[kFixThreads / 32];
  __shared__ double s_best;
  __shared__ int s_bi;
  const int b = blockIdx.x;
  if (!st[b].active) return;
  const HLow B = lb[b];
  const int k = st[b].rank, i = st[b].prow, j = st[b].pcol;
  const long ldu = 3L * B.nr, ldv = 3L * B.nc;
  double* U = Up + B.uoff;
  const double* V = Vp + B.voff;
  for (int q = threadIdx.x; q < 3 * k; q += blockDim.x) sv[q % 3][q / 3] = V[(size_t)(q / 3) * ldv + 3 * j + q % 3];
  if (threadIdx.x == 0) {
    // P[a][c] = residual row a at the pivot triangle's column c.  The residual's 3 x 3 block is often
    // nearly rank-deficient after a few steps, so its usable part is chosen by complete pivoting (up
    // to three rank-one terms, as hmatrix/src/hmatrix.cpp:56-60 takes them): index sets I (rows) and
    // J (columns) with P_IJ well conditioned, and the generalised inverse G (3 x 3) with
    // G[J[q]][I[p]] = (P_IJ^-1)[q][p], zero elsewhere, so that C G R = C_J P_IJ^-1 R_I.
    double P[9], W[9];
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) P[3 * a + c] = W[3 * a + c] = V[(size_t)(k + a) * ldv + 3 * j + c];
    double pmax = 0.0;
    for (int q = 0; q < 9; ++q) pmax = fmax(pmax, fabs(P[q]));
    int I[3], J[3], r = 0;
    bool usedr[3] = {false, false, false}, usedc[3] = {false, false, false};
    if (isfinite(pmax) && pmax > 0.0) {
      for (; r < 3; ++r) {
        int ba = -1, bc = -1;
        double bv = 0.0;
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c)
            if (!usedr[a] && !usedc[c] && fabs(W[3 * a + c]) > bv) {
              bv = fabs(W[3 * a + c]);
              ba = a;
              bc = c;
            }
        if (ba < 0 || !(bv > 1e-10 * pmax)) break;
        I[r] = ba;
        J[r] = bc;
        usedr[ba] = usedc[bc] = true;
        const double piv = W[3 * ba + bc];
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c)
            if (!usedr[a] && !usedc[c]) W[3 * a + c] -= W[3 * a + bc] * W[3 * ba + c] / piv;
      }
    }
    for (int q = 0; q < 9; ++q) s_pinv[q] = 0.0;
    s_ok = r > 0;
    if (r == 1) {
      s_pinv[3 * J[0] + I[0]] = 1.0 / P[3 * I[0] + J[0]];
    } else if (r == 2) {
      const double m00 = P[3 * I[0] + J[0]], m01 = P[3 * I[0] + J[1]], m10 = P[3 * I[1] + J[0]],
                   m11 = P[3 * I[1] + J[1]];
      const double id = 1.0 / (m00 * m11 - m01 * m10);
      // M^-1 = [[m11, -m01], [-m10, m00]] / det, rows indexed by J, columns by I
      s_pinv[3 * J[0] + I[0]] = m11 * id;
      s_pinv[3 * J[0] + I[1]] = -m01 * id;
      s_pinv[3 * J[1] + I[0]] = -m10 * id;
      s_pinv[3 * J[1] + I[1]] = m00 * id;
    } else if (r == 3) {
      const double c00 = P[4] * P[8] - P[5] * P[7], c01 = P[5] * P[6] - P[3] * P[8], c02 = P[3] * P[7] - P[4] * P[6];
      const double id = 1.0 / (P[0] * c00 + P[1] * c01 + P[2] * c02);
      // the full inverse, stored as G[c][a] = (P^-1)[c][a]
      s_pinv[0] = c00 * id;
      s_pinv[1] = (P[2] * P[7] - P[1] * P[8]) * id;
      s_pinv[2] = (P[1] * P[5] - P[2] * P[4]) * id;
      s_pinv[3] = c01 * id;
      s_pinv[4] = (P[0] * P[8] - P[2] * P[6]) * id;
      s_pinv[5] = (P[2] * P[3] - P[0] * P[5]) * id;
      s_pinv[6] = c02 * id;
      s_pinv[7] = (P[1] * P[6] - P[0] * P[7]) * id;
      s_pinv[8] = (P[0] * P[4] - P[1] * P[3]) * id;
    }
    for (int q = 0; q < 9; ++q)
      if (!isfinite(s_pinv[q])) s_ok = 0;
  }
  __syncthreads();
  if (!s_ok) {
    if (threadIdx.x == 0) st[b].active = 0;
    return;
  }
  // residual columns, then U_new = C Pinv, and each row triangle's norm for the next pivot
  double best = -1.0;
  int bi = 0x7fffffff;
  double uu[6] = {0, 0, 0, 0, 0, 0};  // U_new^T U_new (upper triangle)
  for (int t = threadIdx.x; t < B.nr; t += blockDim.x) {
    double nrm = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int row = 3 * t + a;
      double cr[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) cr[c] = U[(size_t)(k + c) * ldu + row];
      for (int q = 0; q < k; ++q) {
        const double u = U[(size_t)q * ldu + row];
#pragma unroll
        for (int c = 0; c < 3; ++c) cr[c] -= u * sv[c][q];
      }
      double un[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) un[c] = cr[0] * s_pinv[c] + cr[1] * s_pinv[3 + c] + cr[2] * s_pinv[6 + c];
#pragma unroll
      for (int c = 0; c < 3; ++c) U[(size_t)(k + c) * ldu + row] = un[c];
      uu[0] += un[0] * un[0];
      uu[1] += un[0] * un[1];
      uu[2] += un[0] * un[2];
      uu[3] += un[1] * un[1];
      uu[4] += un[1] * un[2];
      uu[5] += un[2] * un[2];
      nrm += un[0] * un[0] + un[1] * un[1] + un[2] * un[2];
    }
    // the pivot row's own rows of C P^-1 are the identity: never the next pivot
    if (t != i && nrm > best) {
      best = nrm;
      bi = t;
    }
  }
  double vv[6] = {0, 0, 0, 0, 0, 0};  // V_new^T V_new
  for (int r = threadIdx.x; r < 3 * B.nc; r += blockDim.x) {
    const double v0 = V[(size_t)k * ldv + r], v1 = V[(size_t)(k + 1) * ldv + r], v2 = V[(size_t)(k + 2) * ldv + r];
    vv[0] += v0 * v0;
    vv[1] += v0 * v1;
    vv[2] += v0 * v2;
    vv[3] += v1 * v1;
    vv[4] += v1 * v2;
    vv[5] += v2 * v2;
  }
  // block sums of uu and vv
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double a = uu[q], c = vv[q];
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if (l == 0) {
      s_red[w][q] = a;
      s_red[w][6 + q] = c;
    }
  }
  __syncthreads();  // U_new complete (global writes of this block visible to it after the barrier)
  // cross terms: for each old term q, (U_q . U_new_c)(V_new_c . V_q) summed over c: a warp per q
  for (int q = w; q < k; q += kFixThreads / 32) {
    double du[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
    for (int r = l; r < 3 * B.nr; r += 32) {
      const double u = U[(size_t)q * ldu + r];
#pragma unroll
      for (int c = 0; c < 3; ++c) du[c] += u * U[(size_t)(k + c) * ldu + r];
    }
    for (int r = l; r < 3 * B.nc; r += 32) {
      const double v = V[(size_t)q * ldv + r];
#pragma unroll
      for (int c = 0; c < 3; ++c) dv[c] += v * V[(size_t)(k + c) * ldv + r];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
      for (int o = 16; o > 0; o >>= 1) {
        du[c] += __shfl_down_sync(0xffffffffu, du[c], o);
        dv[c] += __shfl_down_sync(0xffffffffu, dv[c], o);
      }
    if (l == 0) s_cross[q] = du[0] * dv[0] + du[1] * dv[1] + du[2] * dv[2];
  }
  block_argmax<kFixThreads>(best, bi, s_v, s_i, &s_best, &s_bi);
  if (threadIdx.x == 0) {
    double su6[6] = {0, 0, 0, 0, 0, 0}, sv6[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < kFixThreads / 32; ++q)
      for (int c = 0; c < 6; ++c) {
        su6[c] += s_red[q][c];
        sv6[c] += s_red[q][6 + c];
      }
    // trace(uu vv) with both symmetric: diagonal products plus twice the off-diagonal ones
    const double dnorm2 = su6[0] * sv6[0] + su6[3] * sv6[3] + su6[5] * sv6[5] +
                          2.0 * (su6[1] * sv6[1] + su6[2] * sv6[2] + su6[4] * sv6[4]);
    double cross = 0.0;
    for (int q = 0; q < k; ++q) cross += s_cross[q];
    AcaState S = st[b];
    S.norm2 = S.norm2 + dnorm2 + 2.0 * cross;
    S.rank = k + 3;
    const bool small = dnorm2 <= eps * eps * fabs(S.norm2);
    if (small || !isfinite(S.norm2)) S.active = 0;
    else if (S.rank + 3 > B.kcap) {
      S.active = 0;
      S.capped = 1;
    } else if (!(s_best > 0.0)) {
      S.active = 0;
    } else {
      S.prow = s_bi;
    }
    st[b] = S;
  }
}

// Rows and columns of earlier pivots are not excluded beyond the current row: the cross
// approximation reproduces them exactly, so their residuals are zero up to rounding.

// Product, first part: t[toff + j, c] = V[:, j]^T xt[3 c0 .., c] for every term of every low-rank
// block.  One CTA per block, each warp four terms at a time (four independent loads of V per lane),
// the columns of x in passes of eight; the block's rows of x are read through L1 by all its warps.
constexpr int kVtThreads = 128;
template <int QC>
__global__ void __launch_bounds__(kVtThreads)
    k_lr_vt(const HLow* __restrict__ lb, const double* __restrict__ Vp, const double* __restrict__ xt, long ldx,
            int nq, double* __restrict__ tbuf) {
  const HLow B = lb[blockIdx.x];
  const int kr = B.kcap;  // after the fill, the block's rank
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const long ldv = 3L * B.nc;
  const int rows = 3 * B.nc;
  const double* x = xt + 3L * B.c0;
  for (int j0 = 4 * w; j0 < kr; j0 += 4 * (kVtThreads / 32)) {
    const double* v = Vp + B.voff + (size_t)j0 * ldv;
    const int nj = min(4, kr - j0);
    for (int c0 = 0; c0 < nq; c0 += QC) {
      const int qc = min(QC, nq - c0);
      double acc[4][QC];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < QC; ++c) acc[a][c] = 0.0;
      int r = l;
      for (; r + 32 < rows; r += 64) {  // two rows per lane in flight
        double vr[2][4];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int a = 0; a < 4; ++a) vr[h][a] = a < nj ? __ldg(v + (size_t)a * ldv + r + 32 * h) : 0.0;
#pragma unroll
        for (int c = 0; c < QC; ++c)
          if (c < qc) {
            const double x0 = __ldg(x + (size_t)(c0 + c) * ldx + r), x1 = __ldg(x + (size_t)(c0 + c) * ldx + r + 32);
#pragma unroll
            for (int a = 0; a < 4; ++a) acc[a][c] += vr[0][a] * x0 + vr[1][a] * x1;
          }
      }
      for (; r < rows; r += 32) {
        double vr[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) vr[a] = a < nj ? __ldg(v + (size_t)a * ldv + r) : 0.0;
#pragma unroll
        for (int c = 0; c < QC; ++c)
          if (c < qc) {
            const double xv = __ldg(x + (size_t)(c0 + c) * ldx + r);
#pragma unroll
            for (int a = 0; a < 4; ++a) acc[a][c] += vr[a] * xv;
          }
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < QC; ++c) {
          double t = acc[a][c];
          for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
          if (l == 0 && a < nj && c < qc) tbuf[(size_t)(B.toff + j0 + a) * kHQ + c0 + c] = t;
        }
    }
  }
}

// Deflation sums s[c][q] = gdef_c sum over comp == c of xmu . x (one CTA per (surface, column)).
__global__ void k_defl_sums(int n, int ndef, const double* __restrict__ gdef, const double* __restrict__ xmu_t,
                            const int* __restrict__ comp_t, const double* __restrict__ xt, long ldx,
                            double* __restrict__ sdef) {
  const int c = blockIdx.x + 1, q = blockIdx.y;
  __shared__ double red[256 / 32];
  double a = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    if (ndef > 1 && comp_t[k] != c) continue;
    const double* x = xt + (size_t)q * ldx + 3 * (size_t)k;
    a += xmu_t[3 * (size_t)k] * x[0] + xmu_t[3 * (size_t)k + 1] * x[1] + xmu_t[3 * (size_t)k + 2] * x[2];
  }
  for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 256 / 32; ++w) s += red[w];
    sdef[(size_t)(c - 1) * kHQ + q] = gdef[c - 1] * s;
  }
}

constexpr int kLeafThreads = 3 * kHMaxLeaf;  // the most threads per CTA (one per row of the largest leaf)
constexpr int kColChunk = 128;               // source triangles of x staged at a time
constexpr int kSegments = 8;                 // CTAs per leaf row cluster in the product

// Product, second part: CTA (leaf L, segment g) sums the rows of L of every g-th of L's blocks (dense:
// rows times x; low-rank: rows of U times that block's t) into part[g]; four independent loads per
// thread in flight, and kSegments CTAs per leaf, to keep enough bytes moving.
template <int NQ>
__global__ void __launch_bounds__(kLeafThreads)
    k_leaf_mv(const HLeaf* __restrict__ leaves, const HEntry* __restrict__ dent, const HEntry* __restrict__ lent,
              const HDense* __restrict__ db, const HLow* __restrict__ lb, const double* __restrict__ Dp,
              const double* __restrict__ Up, const double* __restrict__ xt, long ldx, const double* __restrict__ tbuf,
              int nq, double* __restrict__ part, long ldp) {
  extern __shared__ double sx[];  // max(3 kColChunk, kHMaxRank) * kHQ
  const HLeaf L = leaves[blockIdx.x];
  const int g = blockIdx.y;
  const int row = threadIdx.x;
  const int m = 3 * L.cnt;
  double acc[NQ];
#pragma unroll
  for (int c = 0; c < NQ; ++c) acc[c] = 0.0;
  for (int e = L.d0 + g; e < L.d1; e += kSegments) {
    const HEntry E = dent[e];
    const HDense B = db[E.blk];
    const long ld = 3L * B.nr;
    const double* A = Dp + B.off + E.rowoff;
    for (int c0 = 0; c0 < B.nc; c0 += kColChunk) {
      const int cn = min(kColChunk, B.nc - c0);
      __syncthreads();
      for (int q = threadIdx.x; q < 3 * cn * nq; q += blockDim.x) {
        const int c = q / (3 * cn), r = q % (3 * cn);
        sx[r * kHQ + c] = xt[(size_t)c * ldx + 3L * (B.c0 + c0) + r];
      }
      __syncthreads();
      if (row < m) {
        const double* a = A + 3L * c0 * ld + row;
        const int rn = 3 * cn;  // a multiple of 3; the tail of fewer than 4 rows below
        int r = 0;
        for (; r + 4 <= rn; r += 4) {
          const double a0 = __ldg(a + (size_t)r * ld), a1 = __ldg(a + (size_t)(r + 1) * ld);
          const double a2 = __ldg(a + (size_t)(r + 2) * ld), a3 = __ldg(a + (size_t)(r + 3) * ld);
#pragma unroll
          for (int c = 0; c < NQ; ++c) {
              acc[c] += a0 * sx[r * kHQ + c];
              acc[c] += a1 * sx[(r + 1) * kHQ + c];
              acc[c] += a2 * sx[(r + 2) * kHQ + c];
              acc[c] += a3 * sx[(r + 3) * kHQ + c];
            }
        }
        for (; r < rn; ++r) {
          const double av = __ldg(a + (size_t)r * ld);
#pragma unroll
          for (int c = 0; c < NQ; ++c) acc[c] += av * sx[r * kHQ + c];
        }
      }
    }
  }
  for (int e = L.l0 + g; e < L.l1; e += kSegments) {
    const HEntry E = lent[e];
    const HLow B = lb[E.blk];
    const long ld = 3L * B.nr;
    __syncthreads();
    const int kr = B.kcap;  // after the fill, the block's rank
    for (int q = threadIdx.x; q < kr * nq; q += blockDim.x) {
      const int j = q / nq, c = q % nq;
      sx[j * kHQ + c] = tbuf[(size_t)(B.toff + j) * kHQ + c];
    }
    __syncthreads();
    if (row < m) {
      const double* u = Up + B.uoff + E.rowoff + row;
      int j = 0;
      for (; j + 4 <= kr; j += 4) {
        const double u0 = __ldg(u + (size_t)j * ld), u1 = __ldg(u + (size_t)(j + 1) * ld);
        const double u2 = __ldg(u + (size_t)(j + 2) * ld), u3 = __ldg(u + (size_t)(j + 3) * ld);
#pragma unroll
        for (int c = 0; c < NQ; ++c) {
            acc[c] += u0 * sx[j * kHQ + c];
            acc[c] += u1 * sx[(j + 1) * kHQ + c];
            acc[c] += u2 * sx[(j + 2) * kHQ + c];
            acc[c] += u3 * sx[(j + 3) * kHQ + c];
          }
      }
      for (; j < kr; ++j) {
        const double uv = __ldg(u + (size_t)j * ld);
#pragma unroll
        for (int c = 0; c < NQ; ++c) acc[c] += uv * sx[j * kHQ + c];
      }
    }
  }
  if (row >= m) return;
  const size_t gr = 3L * L.beg + row;
#pragma unroll
  for (int c = 0; c < NQ; ++c) part[((size_t)g * nq + c) * ldp + gr] = acc[c];
}

// y = the segments' partial sums in order, plus the deflation term xmu_i s[comp(i)].
__global__ void k_leaf_sum(long n3, int nq, const double* __restrict__ part, long ldp, int ndef,
                           const double* __restrict__ xmu_t, const int* __restrict__ comp_t,
                           const double* __restrict__ sdef, double* __restrict__ yt, long ldy) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3 * nq) return;
  const int c = (int)(i / n3);
  const long r = i % n3;
  double a = part[(size_t)c * ldp + r];
#pragma unroll
  for (int g = 1; g < kSegments; ++g) a += part[((size_t)g * nq + c) * ldp + r];
  if (ndef > 0) {
    const int comp = ndef > 1 ? comp_t[r / 3] : 1;
    if (comp >= 1 && comp <= ndef) a += xmu_t[r] * sdef[(size_t)(comp - 1) * kHQ + c];
  }
  yt[(size_t)c * ldy + r] = a;
}

// Block-Jacobi preconditioner apply: z_L = inv_L r_L for every leaf (tree order).
__global__ void __launch_bounds__(kLeafThreads)
    k_bj_apply(const HLeaf* __restrict__ leaves, const double* __restrict__ inv, const double* __restrict__ r, long ldr,
               int nq, double* __restrict__ z, long ldz) {
  extern __shared__ double sx[];  // 3 kHMaxLeaf * kHQ
  const HLeaf L = leaves[blockIdx.x];
  const int m = 3 * L.cnt, row = threadIdx.x;
  for (int q = threadIdx.x; q < m * nq; q += blockDim.x) {
    const int c = q / m, rr = q % m;
    sx[rr * kHQ + c] = r[(size_t)c * ldr + 3L * L.beg + rr];
  }
  __syncthreads();
  if (row >= m) return;
  double acc[kHQ];
#pragma unroll
  for (int c = 0; c < kHQ; ++c) acc[c] = 0.0;
  const double* A = inv + L.inv + row;
  int cc = 0;
  for (; cc + 4 <= m; cc += 4) {
    const double a0 = __ldg(A + (size_t)cc * m), a1 = __ldg(A + (size_t)(cc + 1) * m);
    const double a2 = __ldg(A + (size_t)(cc + 2) * m), a3 = __ldg(A + (size_t)(cc + 3) * m);
#pragma unroll
    for (int c = 0; c < kHQ; ++c)
      if (c < nq) {
        acc[c] += a0 * sx[cc * kHQ + c];
        acc[c] += a1 * sx[(cc + 1) * kHQ + c];
        acc[c] += a2 * sx[(cc + 2) * kHQ + c];
        acc[c] += a3 * sx[(cc + 3) * kHQ + c];
      }
  }
  for (; cc < m; ++cc) {
    const double av = __ldg(A + (size_t)cc * m);
#pragma unroll
    for (int c = 0; c < kHQ; ++c)
      if (c < nq) acc[c] += av * sx[cc * kHQ + c];
  }
#pragma unroll
  for (int c = 0; c < kHQ; ++c)
    if (c < nq) z[(size_t)c * ldz + 3L * L.beg + row] = acc[c];
}

// The leaf's diagonal block plus its deflation term, copied into the inverse's storage.
__global__ void k_bj_copy(const HLeaf* __restrict__ leaves, const HDense* __restrict__ db, const double* __restrict__ Dp,
                          int ndef, const double* __restrict__ gdef, const double* __restrict__ xmu_t,
                          const int* __restrict__ comp_t, double* __restrict__ inv) {
  const HLeaf L = leaves[blockIdx.x];
  const HDense B = db[L.diag];
  const int m = 3 * L.cnt;
  for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
    const int r = q % m, c = q / m;
    double v = Dp[B.off + (size_t)c * m + r];
    if (ndef > 0) {
      const int ti = L.beg + r / 3, sj = L.beg + c / 3;
      const int ci = ndef > 1 ? comp_t[ti] : 1, cj = ndef > 1 ? comp_t[sj] : 1;
      if (ci == cj && cj >= 1 && cj <= ndef) v = v + gdef[cj - 1] * xmu_t[3L * L.beg + c] * xmu_t[3L * L.beg + r];
    }
    inv[L.inv + q] = v;
  }
}

constexpr int kGjThreads = 512;

// In-place Gauss-Jordan inversion with partial pivoting of each leaf's block (column-major, m x m):
// after the sweep over PA, the inverse is recovered by swapping columns back in reverse order.
__global__ void __launch_bounds__(kGjThreads) k_bj_invert(const HLeaf* __restrict__ leaves, double* __restrict__ inv,
                                                          int* __restrict__ status) {
  __shared__ double s_col[3 * kHMaxLeaf], s_row[3 * kHMaxLeaf];
  __shared__ int s_piv[3 * kHMaxLeaf];
  __shared__ double s_v[kGjThreads / 32];
  __shared__ int s_i[kGjThreads / 32];
  __shared__ double s_best;
  __shared__ int s_bi;
  const HLeaf L = leaves[blockIdx.x];
  const int m = 3 * L.cnt;
  double* A = inv + L.inv;
  for (int p = 0; p < m; ++p) {
    double best = -1.0;
    int bi = 0x7fffffff;
    for (int r = p + threadIdx.x; r < m; r += blockDim.x) {
      const double v = fabs(A[(size_t)p * m + r]);
      if (v > best) {
        best = v;
        bi = r;
      }
    }
    block_argmax<kGjThreads>(best, bi, s_v, s_i, &s_best, &s_bi);
    if (!(s_best > 0.0) || !isfinite(s_best)) {
      if (threadIdx.x == 0) atomicExch(status, (int)kNotFinite);
      return;  // every thread of the block takes this branch (s_best is shared)
    }
    const int piv = s_bi;
    if (piv != p)
      for (int c = threadIdx.x; c < m; c += blockDim.x) {
        const double t = A[(size_t)c * m + p];
        A[(size_t)c * m + p] = A[(size_t)c * m + piv];
        A[(size_t)c * m + piv] = t;
      }
    __syncthreads();
    const double d = 1.0 / A[(size_t)p * m + p];
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      s_col[r] = A[(size_t)p * m + r];
      s_row[r] = A[(size_t)r * m + p];
    }
    if (threadIdx.x == 0) s_piv[p] = piv;
    __syncthreads();
    // row p scaled (its pivot entry becomes d), the other rows eliminated; column p becomes -col * d
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
      const int r = q % m, c = q / m;
      if (c == p) {
        A[(size_t)c * m + r] = (r == p) ? d : -s_col[r] * d;
      } else {
        const double arow = s_row[c] * d;
        if (r == p) A[(size_t)c * m + r] = arow;
        else A[(size_t)c * m + r] = A[(size_t)c * m + r] - s_col[r] * arow;
      }
    }
    __syncthreads();
  }
  for (int p = m - 1; p >= 0; --p) {
    const int piv = s_piv[p];
    if (piv != p)
      for (int r = threadIdx.x; r < m; r += blockDim.x) {
        const double t = A[(size_t)p * m + r];
        A[(size_t)p * m + r] = A[(size_t)piv * m + r];
        A[(size_t)piv * m + r] = t;
      }
    __syncthreads();
  }
}

// GMRES helpers over nq columns of 3n rows (column stride n3 for every vector block).
__global__ void k_gather_rows(int n, const int* __restrict__ perm, const double* __restrict__ x, long ldx, int nq,
                              double* __restrict__ xt, long ldt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3L * n * nq) return;
  const int c = (int)(i / (3L * n));
  const long r = i % (3L * n);
  xt[(size_t)c * ldt + r] = x[(size_t)c * ldx + 3L * perm[r / 3] + r % 3];
}

__global__ void k_scatter_rows(int n, const int* __restrict__ perm, const double* __restrict__ xt, long ldt, int nq,
                               double* __restrict__ x, long ldx) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3L * n * nq) return;
  const int c = (int)(i / (3L * n));
  const long r = i % (3L * n);
  x[(size_t)c * ldx + 3L * perm[r / 3] + r % 3] = xt[(size_t)c * ldt + r];
}

// out[j * nq + c] = V_j[:, c] . W[:, c] (V_j = V + j nq n3), a CTA per (j, c)
__global__ void k_dots(long n3, int nq, const double* __restrict__ V, const double* __restrict__ W,
                       double* __restrict__ out) {
  const int j = blockIdx.x, c = blockIdx.y;
  const double* v = V + ((size_t)j * nq + c) * n3;
  const double* w = W + (size_t)c * n3;
  __shared__ double red[8];
  double a = 0.0;
  for (long r = threadIdx.x; r < n3; r += blockDim.x) a += v[r] * w[r];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int q = 0; q < 8; ++q) s += red[q];
    out[(size_t)j * nq + c] = s;
  }
}

// W[:, c] -= sum_j h[j nq + c] V_j[:, c]   (sign = -1), or Z[:, c] = sum_j h V_j (sign = 0)
__global__ void k_combine(long n3, int nq, int nj, const double* __restrict__ V, const double* __restrict__ h,
                          double* __restrict__ W, int subtract) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3 * nq) return;
  const int c = (int)(i / n3);
  const long r = i % n3;
  double a = 0.0;
  for (int j = 0; j < nj; ++j) a += h[(size_t)j * nq + c] * V[((size_t)j * nq + c) * n3 + r];
  if (subtract) W[(size_t)c * n3 + r] -= a;
  else W[(size_t)c * n3 + r] = a;
}

// V_next[:, c] = W[:, c] / nrm[c] (zero when nrm is zero); also R = B - W for the residual (mode 1)
__global__ void k_scale(long n3, int nq, const double* __restrict__ W, const double* __restrict__ nrm,
                        double* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3 * nq) return;
  const int c = (int)(i / n3);
  const double s = nrm[c];
  out[i] = s > 0.0 ? W[i] / s : 0.0;
}

__global__ void k_sub(long count, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) out[i] = a[i] - b[i];
}

__global__ void k_add(long count, const double* __restrict__ a, double* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) out[i] += a[i];
}

void hck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw std::runtime_error(std::string("H-matrix: ") + what + ": " + cudaGetErrorString(e));
  }
}

unsigned blocks_for(long count, int threads) { return (unsigned)((count + threads - 1) / threads); }

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  ~Buf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void ensure(size_t need, const char* what) {
    if (p && bytes >= need) return;
    reset();
    if (need == 0) need = 16;
    if (cudaMalloc(&p, need) != cudaSuccess) {
      cudaGetLastError();
      size_t fr = 0, tot = 0;
      cudaMemGetInfo(&fr, &tot);
      throw std::runtime_error(std::string("H-matrix: cannot allocate ") + what + ": " + std::to_string(need / 1e9) +
                               " GB needed, " + std::to_string(fr / 1e9) + " GB free on the GPU");
    }
    bytes = need;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

template <class T>
void upload(Buf& b, const std::vector<T>& v, const char* what, cudaStream_t s) {
  b.ensure(sizeof(T) * std::max<size_t>(1, v.size()), what);
  if (!v.empty()) hck(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s), what);
}

}  // namespace

struct HMatrixSolver::Impl {
  int leaf = 128, kmax = 90;
  double eta = 2.0, eps = 1e-4;
  int n = 0, ndef = 0;
  double cg = 1.0;
  HPlan plan;
  std::vector<HDense> dense;
  std::vector<HLow> low;
  std::vector<HLeaf> leaves;
  int nterms = 0, capped = 0, max_rank = 0;
  double dense_entries = 0, low_entries = 0, mean_rank = 0;
  double ms_fill = 0, ms_aca = 0, ms_pre = 0;
  HReport last;
  Buf perm, geo_t, xc_t, self9_t, xmu_t, comp_t, gdef;
  Buf d_dense, d_low, d_leaves, d_dent, d_lent, d_dtile, d_rtile, d_ctile, d_state, status;
  Buf D, Up, Vp, inv;
  Buf xt, yt, tb, sdef, part;         // product scratch
  int threads = kLeafThreads;         // CTA size of the per-leaf kernels: 3 x the largest leaf, rounded up to 32
  Buf gV, gW, gZ, gX, gR, gB, gh, gn;  // GMRES
  size_t held() const {
    size_t s = 0;
    for (const Buf* b : {&perm, &geo_t, &xc_t, &self9_t, &xmu_t, &comp_t, &gdef, &d_dense, &d_low, &d_leaves, &d_dent,
                         &d_lent, &d_dtile, &d_rtile, &d_ctile, &d_state, &status, &D, &Up, &Vp, &inv, &xt, &yt,
                         &tb, &sdef, &part, &gV, &gW, &gZ, &gX, &gR, &gB, &gh, &gn})
      s += b->bytes;
    return s;
  }

  // y_t = (H + deflation) x_t, both in tree order (column stride ld)
  void apply_tree(int nq, const double* x, long ldx, double* y, long ldy, cudaStream_t s) {
    if (nterms > 0) {
      auto vt = nq >= 8 ? k_lr_vt<8> : nq == 7 ? k_lr_vt<7> : nq == 6 ? k_lr_vt<6> : nq == 5 ? k_lr_vt<5>
              : nq == 4 ? k_lr_vt<4> : nq == 3 ? k_lr_vt<3> : nq == 2 ? k_lr_vt<2> : k_lr_vt<1>;
      vt<<<(unsigned)low.size(), kVtThreads, 0, s>>>(d_low.as<HLow>(), Vp.as<double>(), x, ldx, nq, tb.as<double>());
      BGPU_COUNT_LAUNCH();
    }
    if (ndef > 0) {
      k_defl_sums<<<dim3(ndef, nq), 256, 0, s>>>(n, ndef, gdef.as<double>(), xmu_t.as<double>(), comp_t.as<int>(), x,
                                                 ldx, sdef.as<double>());
      BGPU_COUNT_LAUNCH();
    }
    const size_t smem = sizeof(double) * std::max(3 * kColChunk, kHMaxRank) * kHQ;
    const long n3 = 3L * n;
    decltype(&k_leaf_mv<1>) mv = nullptr;
    switch (nq) {
#define BGPU_HQ_CASE(q) \
  case q:               \
    mv = k_leaf_mv<q>;  \
    break;
      BGPU_HQ_CASE(1) BGPU_HQ_CASE(2) BGPU_HQ_CASE(3) BGPU_HQ_CASE(4) BGPU_HQ_CASE(5) BGPU_HQ_CASE(6)
      BGPU_HQ_CASE(7) BGPU_HQ_CASE(8) BGPU_HQ_CASE(9) BGPU_HQ_CASE(10) BGPU_HQ_CASE(11) BGPU_HQ_CASE(12)
      BGPU_HQ_CASE(13) BGPU_HQ_CASE(14) BGPU_HQ_CASE(15) BGPU_HQ_CASE(16)
#undef BGPU_HQ_CASE
      default:
        throw std::runtime_error("H-matrix: 1 to 16 columns per product");
    }
    mv<<<dim3((unsigned)leaves.size(), kSegments), threads, smem, s>>>(
        d_leaves.as<HLeaf>(), d_dent.as<HEntry>(), d_lent.as<HEntry>(), d_dense.as<HDense>(), d_low.as<HLow>(),
        D.as<double>(), Up.as<double>(), x, ldx, tb.as<double>(), nq, part.as<double>(), n3);
    BGPU_COUNT_LAUNCH();
    k_leaf_sum<<<blocks_for(n3 * nq, 256), 256, 0, s>>>(n3, nq, part.as<double>(), n3, ndef, xmu_t.as<double>(),
                                                        comp_t.as<int>(), sdef.as<double>(), y, ldy);
    BGPU_COUNT_LAUNCH();
    hck(cudaGetLastError(), "product");
  }

  void precond(int nq, const double* r, long ldr, double* z, long ldz, cudaStream_t s) {
    const size_t smem = sizeof(double) * 3 * kHMaxLeaf * kHQ;
    k_bj_apply<<<(unsigned)leaves.size(), threads, smem, s>>>(d_leaves.as<HLeaf>(), inv.as<double>(), r, ldr, nq, z,
                                                                   ldz);
    BGPU_COUNT_LAUNCH();
    hck(cudaGetLastError(), "preconditioner");
  }
};

HMatrixSolver::HMatrixSolver() : p_(new Impl) {}
HMatrixSolver::~HMatrixSolver() { delete p_; }

void HMatrixSolver::set_options(int leaf, double eta, int kmax) {
  if (leaf < 8 || leaf > kHMaxLeaf) throw std::runtime_error("H-matrix: leaf size must be in [8, 128]");
  if (!(eta > 0.0)) throw std::runtime_error("H-matrix: eta must be positive");
  if (kmax < 3 || kmax > kHMaxRank || kmax % 3) throw std::runtime_error("H-matrix: kmax must be a multiple of 3 in [3, 120]");
  p_->leaf = leaf;
  p_->eta = eta;
  p_->kmax = kmax;
}

void HMatrixSolver::build(const DevMesh& m, const DevDeflation& d, int ndef, double eps, cudaStream_t s) {
  Impl& I = *p_;
  I.n = m.n;
  I.cg = m.cg;
  I.eps = (eps > 0.0 && eps < 1.0) ? eps : 1e-4;
  I.ndef = std::max(0, ndef);
  if (I.ndef > 256) throw std::runtime_error("H-matrix: at most 256 surfaces (deflation terms)");
  const int n = m.n;
  // host copies of the corners and incenters for the plan
  std::vector<double> geo((size_t)n * kGeoStride), xc((size_t)n * kXcStride);
  hck(cudaMemcpyAsync(geo.data(), m.geo, geo.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "geometry copy");
  hck(cudaMemcpyAsync(xc.data(), m.xc, xc.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "incenter copy");
  hck(cudaStreamSynchronize(s), "geometry copy");
  I.plan = hplan_build(n, geo.data(), xc.data(), I.leaf, I.eta, I.kmax);
  const HPlan& P = I.plan;
  // block lists
  I.dense.clear();
  I.low.clear();
  std::vector<int> dense_of_leaf(P.cl.size(), -1);
  long long doff = 0, uoff = 0, voff = 0;
  std::vector<std::vector<HEntry>> dent(P.cl.size()), lent(P.cl.size());
  std::vector<int> leaf_index(P.cl.size(), -1);
  for (size_t q = 0; q < P.leaves.size(); ++q) leaf_index[P.leaves[q]] = (int)q;
  for (const HPlan::Block& b : P.blocks) {
    const HPlan::Cluster &ct = P.cl[b.t], &cs = P.cl[b.s];
    if (!b.lowrank) {
      HDense D{ct.beg, ct.cnt, cs.beg, cs.cnt, doff};
      doff += 9LL * ct.cnt * cs.cnt;
      if (b.t == b.s) dense_of_leaf[b.t] = (int)I.dense.size();
      I.dense.push_back(D);
    } else {
      HLow L{ct.beg, ct.cnt, cs.beg, cs.cnt, uoff, voff, std::min(I.kmax, 3 * std::min(ct.cnt, cs.cnt)), 0};
      L.kcap -= L.kcap % 3;
      uoff += 3LL * ct.cnt * L.kcap;
      voff += 3LL * cs.cnt * L.kcap;
      I.low.push_back(L);
    }
  }
  // per-leaf row lists: every block whose row cluster contains the leaf
  I.leaves.clear();
  std::vector<HEntry> de, le;
  {
    // the leaves a cluster covers are contiguous in tree order: [first, first + count)
    std::vector<int> first(P.cl.size()), count(P.cl.size());
    for (size_t c = P.cl.size(); c-- > 0;) {
      if (P.cl[c].son0 < 0) {
        first[c] = leaf_index[c];
        count[c] = 1;
      } else {
        first[c] = first[P.cl[c].son0];
        count[c] = count[P.cl[c].son0] + count[P.cl[c].son0 + 1];
      }
    }
    std::vector<std::vector<HEntry>> dl(P.leaves.size()), ll(P.leaves.size());
    int di = 0, li = 0;
    for (const HPlan::Block& b : P.blocks) {
      const int f = first[b.t], c = count[b.t];
      for (int q = f; q < f + c; ++q) {
        const HEntry e{b.lowrank ? li : di, 3 * (P.cl[P.leaves[q]].beg - P.cl[b.t].beg)};
        (b.lowrank ? ll : dl)[q].push_back(e);
      }
      (b.lowrank ? li : di)++;
    }
    long long ioff = 0;
    for (size_t q = 0; q < P.leaves.size(); ++q) {
      const HPlan::Cluster& c = P.cl[P.leaves[q]];
      if (c.cnt > kHMaxLeaf) throw std::runtime_error("H-matrix: leaf larger than 128 triangles");
      HLeaf L{c.beg, c.cnt, (int)de.size(), 0, (int)le.size(), 0, ioff, dense_of_leaf[P.leaves[q]], 0};
      if (L.diag < 0) throw std::runtime_error("H-matrix: a leaf has no diagonal block");
      de.insert(de.end(), dl[q].begin(), dl[q].end());
      le.insert(le.end(), ll[q].begin(), ll[q].end());
      L.d1 = (int)de.size();
      L.l1 = (int)le.size();
      ioff += 9LL * c.cnt * c.cnt;
      I.leaves.push_back(L);
    }
    I.inv.ensure(sizeof(double) * (size_t)std::max(1LL, ioff), "block-Jacobi inverses");
  }
  // tile lists
  std::vector<int> dtile, rtile, ctile;
  long tot = 0;
  for (const HDense& D : I.dense) {
    dtile.push_back((int)tot);
    tot += (long)((D.nr + kTgtTile - 1) / kTgtTile) * ((D.nc + kSrcTile - 1) / kSrcTile);
  }
  const long ntile_d = tot;
  long tr = 0, tc = 0;
  for (const HLow& L : I.low) {
    rtile.push_back((int)tr);
    ctile.push_back((int)tc);
    tr += (L.nc + kAcaThreads - 1) / kAcaThreads;
    tc += (L.nr + kAcaThreads - 1) / kAcaThreads;
  }
  if (ntile_d > 0x7fffffffL || tr > 0x7fffffffL || tc > 0x7fffffffL) throw std::runtime_error("H-matrix: too many tiles");
  I.dense_entries = (double)doff;
  // device buffers
  I.perm.ensure(sizeof(int) * n, "tree order");
  hck(cudaMemcpyAsync(I.perm.p, P.perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s), "perm copy");
  I.geo_t.ensure(sizeof(double) * n * kGeoStride, "geometry (tree order)");
  I.xc_t.ensure(sizeof(double) * n * kXcStride, "incenters (tree order)");
  I.self9_t.ensure(sizeof(double) * n * 9, "self blocks (tree order)");
  k_tree_gather<<<blocks_for(n, 128), 128, 0, s>>>(n, I.perm.as<int>(), m.geo, m.xc, m.self9, I.geo_t.as<double>(),
                                                   I.xc_t.as<double>(), I.self9_t.as<double>());
  BGPU_COUNT_LAUNCH();
  I.xmu_t.ensure(sizeof(double) * 3 * n, "deflation vectors (tree order)");
  I.comp_t.ensure(sizeof(int) * n, "surfaces (tree order)");
  I.gdef.ensure(sizeof(double) * std::max(1, I.ndef), "deflation weights");
  if (I.ndef > 0) {
    k_defl_gather<<<blocks_for(n, 128), 128, 0, s>>>(n, I.perm.as<int>(), d.xmu, I.ndef > 1 ? d.comp : nullptr,
                                                     I.xmu_t.as<double>(), I.comp_t.as<int>());
    BGPU_COUNT_LAUNCH();
    hck(cudaMemcpyAsync(I.gdef.p, d.gdef, sizeof(double) * I.ndef, cudaMemcpyDeviceToDevice, s), "gdef copy");
  }
  upload(I.d_dense, I.dense, "dense block list", s);
  upload(I.d_low, I.low, "low-rank block list", s);
  upload(I.d_dtile, dtile, "tile list", s);
  upload(I.d_rtile, rtile, "tile list", s);
  upload(I.d_ctile, ctile, "tile list", s);
  upload(I.d_dent, de, "leaf lists", s);
  upload(I.d_lent, le, "leaf lists", s);
  upload(I.d_leaves, I.leaves, "leaves", s);
  static bool attrs = false;
  if (!attrs) {
    const int smem = (int)(sizeof(double) * std::max(3 * kColChunk, kHMaxRank) * kHQ);
    for (auto f : {k_leaf_mv<1>, k_leaf_mv<2>, k_leaf_mv<3>, k_leaf_mv<4>, k_leaf_mv<5>, k_leaf_mv<6>, k_leaf_mv<7>,
                   k_leaf_mv<8>, k_leaf_mv<9>, k_leaf_mv<10>, k_leaf_mv<11>, k_leaf_mv<12>, k_leaf_mv<13>,
                   k_leaf_mv<14>, k_leaf_mv<15>, k_leaf_mv<16>})
      hck(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "kernel attributes");
    hck(cudaFuncSetAttribute(k_bj_apply, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * 3 * kHMaxLeaf * kHQ)),
        "kernel attributes");
    attrs = true;
  }
  I.status.ensure(64, "status");
  hck(cudaMemsetAsync(I.status.p, 0, 64, s), "status clear");
  I.D.ensure(sizeof(double) * (size_t)std::max(1LL, doff), "dense blocks");
  I.Up.ensure(sizeof(double) * (size_t)std::max(1LL, uoff), "low-rank factors U");
  I.Vp.ensure(sizeof(double) * (size_t)std::max(1LL, voff), "low-rank factors V");
  cudaEvent_t e0, e1, e2, e3;
  hck(cudaEventCreate(&e0), "event");
  hck(cudaEventCreate(&e1), "event");
  hck(cudaEventCreate(&e2), "event");
  hck(cudaEventCreate(&e3), "event");
  hck(cudaEventRecord(e0, s), "event");
  // near field
  if (ntile_d > 0) {
    k_fill_dense<<<(unsigned)ntile_d, kTgtTile, 0, s>>>(I.d_dense.as<HDense>(), I.d_dtile.as<int>(), (int)I.dense.size(),
                                                        I.geo_t.as<double>(), I.xc_t.as<double>(), I.self9_t.as<double>(),
                                                        m.cg, I.D.as<double>());
    BGPU_COUNT_LAUNCH();
    hck(cudaGetLastError(), "dense fill");
  }
  hck(cudaEventRecord(e1, s), "event");
  // far field: batched cross approximation
  const int nlb = (int)I.low.size();
  std::vector<AcaState> st(nlb);
  for (auto& a : st) {
    a = AcaState{};
    a.active = 1;
  }
  upload(I.d_state, st, "ACA state", s);
  for (int step = 0; step < I.kmax / 3 && nlb > 0; ++step) {
    k_aca_rows<<<(unsigned)tr, kAcaThreads, 0, s>>>(I.d_low.as<HLow>(), I.d_rtile.as<int>(), nlb, I.d_state.as<AcaState>(),
                                                   I.geo_t.as<double>(), I.xc_t.as<double>(), I.self9_t.as<double>(),
                                                   m.cg, I.Vp.as<double>());
    BGPU_COUNT_LAUNCH();
    k_aca_row_fix<<<nlb, kFixThreads, 0, s>>>(I.d_low.as<HLow>(), I.d_state.as<AcaState>(), I.Up.as<double>(),
                                              I.Vp.as<double>());
    BGPU_COUNT_LAUNCH();
    k_aca_cols<<<(unsigned)tc, kAcaThreads, 0, s>>>(I.d_low.as<HLow>(), I.d_ctile.as<int>(), nlb, I.d_state.as<AcaState>(),
                                                   I.geo_t.as<double>(), I.xc_t.as<double>(), I.self9_t.as<double>(),
                                                   m.cg, I.Up.as<double>());
    BGPU_COUNT_LAUNCH();
    k_aca_col_fix<<<nlb, kFixThreads, 0, s>>>(I.d_low.as<HLow>(), I.d_state.as<AcaState>(), I.eps, I.Up.as<double>(),
                                              I.Vp.as<double>());
    BGPU_COUNT_LAUNCH();
    hck(cudaGetLastError(), "cross approximation");
    if (step % 4 == 3) {
      hck(cudaMemcpyAsync(st.data(), I.d_state.p, sizeof(AcaState) * nlb, cudaMemcpyDeviceToHost, s), "ACA state");
      hck(cudaStreamSynchronize(s), "cross approximation");
      bool any = false;
      for (const auto& a : st) any = any || a.active;
      if (!any) break;
    }
  }
  hck(cudaEventRecord(e2, s), "event");
  hck(cudaMemcpyAsync(st.data(), I.d_state.p, sizeof(AcaState) * std::max(0, nlb), cudaMemcpyDeviceToHost, s),
      "ACA state");
  hck(cudaStreamSynchronize(s), "cross approximation");
  // final ranks into the block list (kcap := rank), product term list
  int nterms = 0;
  I.capped = 0;
  I.max_rank = 0;
  I.low_entries = 0;
  long long rsum = 0;
  for (int b = 0; b < nlb; ++b) {
    HLow& L = I.low[b];
    const int r = st[b].rank;
    L.toff = nterms;
    L.kcap = r;
    nterms += r;
    I.capped += st[b].capped;
    I.max_rank = std::max(I.max_rank, r);
    rsum += r;
    I.low_entries += 3.0 * (L.nr + L.nc) * r;
  }
  I.mean_rank = nlb ? (double)rsum / nlb : 0.0;
  I.nterms = nterms;
  upload(I.d_low, I.low, "low-rank block list", s);
  // block-Jacobi preconditioner
  k_bj_copy<<<(unsigned)I.leaves.size(), 256, 0, s>>>(I.d_leaves.as<HLeaf>(), I.d_dense.as<HDense>(), I.D.as<double>(),
                                                       I.ndef, I.gdef.as<double>(), I.xmu_t.as<double>(),
                                                       I.comp_t.as<int>(), I.inv.as<double>());
  BGPU_COUNT_LAUNCH();
  k_bj_invert<<<(unsigned)I.leaves.size(), kGjThreads, 0, s>>>(I.d_leaves.as<HLeaf>(), I.inv.as<double>(),
                                                               I.status.as<int>());
  BGPU_COUNT_LAUNCH();
  hck(cudaGetLastError(), "preconditioner");
  hck(cudaEventRecord(e3, s), "event");
  // product scratch
  I.tb.ensure(sizeof(double) * (size_t)std::max(1, I.nterms) * kHQ, "product terms");
  I.sdef.ensure(sizeof(double) * (size_t)std::max(1, I.ndef) * kHQ, "deflation sums");
  I.part.ensure(sizeof(double) * 3 * (size_t)n * kHQ * kSegments, "product partial sums");
  {
    int mx = 1;
    for (const HLeaf& L : I.leaves) mx = std::max(mx, L.cnt);
    I.threads = std::min(kLeafThreads, (3 * mx + 31) / 32 * 32);
  }
  int stv = 0;
  hck(cudaMemcpyAsync(&stv, I.status.p, sizeof(int), cudaMemcpyDeviceToHost, s), "status");
  hck(cudaStreamSynchronize(s), "H-matrix build");
  float t1 = 0, t2 = 0, t3 = 0;
  cudaEventElapsedTime(&t1, e0, e1);
  cudaEventElapsedTime(&t2, e1, e2);
  cudaEventElapsedTime(&t3, e2, e3);
  I.ms_fill = t1;
  I.ms_aca = t2;
  I.ms_pre = t3;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  cudaEventDestroy(e3);
  if (stv != 0) throw std::runtime_error("H-matrix: a diagonal block of the preconditioner is singular");
}

void HMatrixSolver::matvec(int nrhs, const double* d_x, long ldx, double* d_y, long ldy, cudaStream_t s) {
  Impl& I = *p_;
  const long n3 = 3L * I.n;
  for (int c = 0; c < nrhs; c += kHQ) {
    const int q = std::min(kHQ, nrhs - c);
    I.xt.ensure(sizeof(double) * n3 * kHQ, "product vectors");
    I.yt.ensure(sizeof(double) * n3 * kHQ, "product vectors");
    k_gather_rows<<<blocks_for(n3 * q, 256), 256, 0, s>>>(I.n, I.perm.as<int>(), d_x + (size_t)c * ldx, ldx, q,
                                                          I.xt.as<double>(), n3);
    BGPU_COUNT_LAUNCH();
    I.apply_tree(q, I.xt.as<double>(), n3, I.yt.as<double>(), n3, s);
    k_scatter_rows<<<blocks_for(n3 * q, 256), 256, 0, s>>>(I.n, I.perm.as<int>(), I.yt.as<double>(), n3, q,
                                                           d_y + (size_t)c * ldy, ldy);
    BGPU_COUNT_LAUNCH();
  }
  hck(cudaGetLastError(), "product");
}

void HMatrixSolver::solve(int nrhs, double* d_b, long ldb, cudaStream_t s, HReport* rep) {
  Impl& I = *p_;
  const long n3 = 3L * I.n;
  const int m = 30, maxsteps = 500;  // hmatrix/src/api.cpp:39-40 (restart length, steps per solve)
  const double tol = std::max(0.1 * I.eps, 1e-14);  // api.cpp:41, :840
  HReport out;
  for (int c0 = 0; c0 < nrhs; c0 += kHQ) {
    const int q = std::min(kHQ, nrhs - c0);
    const size_t vec = sizeof(double) * n3 * q;
    I.gV.ensure(vec * (m + 1), "GMRES basis");
    I.gW.ensure(vec, "GMRES vectors");
    I.gZ.ensure(vec, "GMRES vectors");
    I.gX.ensure(vec, "GMRES vectors");
    I.gR.ensure(vec, "GMRES vectors");
    I.gB.ensure(vec, "GMRES vectors");
    I.gh.ensure(sizeof(double) * (2 * (m + 1) + 2) * q, "GMRES coefficients");
    I.gn.ensure(sizeof(double) * (m + 1) * q, "GMRES coefficients");
    double *V = I.gV.as<double>(), *W = I.gW.as<double>(), *Z = I.gZ.as<double>(), *X = I.gX.as<double>();
    double *R = I.gR.as<double>(), *B = I.gB.as<double>(), *h = I.gh.as<double>();
    double* h2 = h + (size_t)(m + 1) * q;
    double* hn = h2 + (size_t)(m + 1) * q;
    const unsigned gb = blocks_for(n3 * q, 256);
    k_gather_rows<<<gb, 256, 0, s>>>(I.n, I.perm.as<int>(), d_b + (size_t)c0 * ldb, ldb, q, B, n3);
    BGPU_COUNT_LAUNCH();
    hck(cudaMemsetAsync(X, 0, vec, s), "GMRES start");
    // ||b||
    std::vector<double> bn(q), beta(q);
    k_dots<<<dim3(1, q), 256, 0, s>>>(n3, q, B, B, hn);
    BGPU_COUNT_LAUNCH();
    hck(cudaMemcpyAsync(bn.data(), hn, sizeof(double) * q, cudaMemcpyDeviceToHost, s), "GMRES norm");
    hck(cudaStreamSynchronize(s), "GMRES");
    for (auto& v : bn) v = std::sqrt(v);
    int steps = 0, restarts = 0;
    double worst = 0.0;
    std::vector<double> hh((size_t)(m + 1) * q * 2 + q);
    for (;;) {
      // true residual R = B - A X (X = 0 on the first pass)
      I.apply_tree(q, X, n3, W, n3, s);
      k_sub<<<gb, 256, 0, s>>>(n3 * q, B, W, R);
      BGPU_COUNT_LAUNCH();
      k_dots<<<dim3(1, q), 256, 0, s>>>(n3, q, R, R, hn);
      BGPU_COUNT_LAUNCH();
      hck(cudaMemcpyAsync(beta.data(), hn, sizeof(double) * q, cudaMemcpyDeviceToHost, s), "GMRES norm");
      hck(cudaStreamSynchronize(s), "GMRES");
      worst = 0.0;
      bool done = true;
      for (int c = 0; c < q; ++c) {
        beta[c] = std::sqrt(beta[c]);
        const double rr = bn[c] > 0 ? beta[c] / bn[c] : 0.0;
        if (!(rr <= worst)) worst = rr;  // a NaN stays
        if (!(rr <= tol)) done = false;
      }
      if (done) break;
      if (steps >= maxsteps || !std::isfinite(worst))
        throw std::runtime_error("H-matrix GMRES did not reach a relative residual of " + std::to_string(tol) + " in " +
                                 std::to_string(steps) + " steps (reached " + std::to_string(worst) + ")");
      ++restarts;
      hck(cudaMemcpyAsync(hn, beta.data(), sizeof(double) * q, cudaMemcpyHostToDevice, s), "GMRES norm");
      k_scale<<<gb, 256, 0, s>>>(n3, q, R, hn, V);
      BGPU_COUNT_LAUNCH();
      // Arnoldi with Givens rotations per column
      std::vector<std::vector<double>> H(q, std::vector<double>((size_t)(m + 1) * m, 0.0));
      std::vector<std::vector<double>> g(q, std::vector<double>(m + 1, 0.0)), cs(q, std::vector<double>(m)),
          sn(q, std::vector<double>(m));
      std::vector<int> jc(q, 0);  // valid steps of each column
      std::vector<char> conv(q, 0);
      for (int c = 0; c < q; ++c) {
        g[c][0] = beta[c];
        conv[c] = !(beta[c] > 0.0);
      }
      int j = 0;
      for (; j < m && steps < maxsteps; ++j) {
        I.precond(q, V + (size_t)j * q * n3, n3, Z, n3, s);
        I.apply_tree(q, Z, n3, W, n3, s);
        k_dots<<<dim3(j + 1, q), 256, 0, s>>>(n3, q, V, W, h);
        BGPU_COUNT_LAUNCH();
        k_combine<<<gb, 256, 0, s>>>(n3, q, j + 1, V, h, W, 1);
        BGPU_COUNT_LAUNCH();
        k_dots<<<dim3(j + 1, q), 256, 0, s>>>(n3, q, V, W, h2);
        BGPU_COUNT_LAUNCH();
        k_combine<<<gb, 256, 0, s>>>(n3, q, j + 1, V, h2, W, 1);
        BGPU_COUNT_LAUNCH();
        k_dots<<<dim3(1, q), 256, 0, s>>>(n3, q, W, W, hn);
        BGPU_COUNT_LAUNCH();
        hck(cudaMemcpyAsync(hh.data(), h, sizeof(double) * ((size_t)2 * (m + 1) * q + q), cudaMemcpyDeviceToHost, s),
            "GMRES coefficients");
        hck(cudaStreamSynchronize(s), "GMRES");
        std::vector<double> nrm(q);
        for (int c = 0; c < q; ++c) nrm[c] = std::sqrt(hh[(size_t)2 * (m + 1) * q + c]);
        hck(cudaMemcpyAsync(hn, nrm.data(), sizeof(double) * q, cudaMemcpyHostToDevice, s), "GMRES norm");
        k_scale<<<gb, 256, 0, s>>>(n3, q, W, hn, V + (size_t)(j + 1) * q * n3);
        BGPU_COUNT_LAUNCH();
        ++steps;
        bool all = true;
        for (int c = 0; c < q; ++c) {
          if (conv[c]) continue;
          std::vector<double>& Hc = H[c];
          for (int i = 0; i <= j; ++i)
            Hc[(size_t)j * (m + 1) + i] = hh[(size_t)i * q + c] + hh[(size_t)(m + 1) * q + (size_t)i * q + c];
          Hc[(size_t)j * (m + 1) + j + 1] = nrm[c];
          for (int i = 0; i < j; ++i) {
            const double a = Hc[(size_t)j * (m + 1) + i], b = Hc[(size_t)j * (m + 1) + i + 1];
            Hc[(size_t)j * (m + 1) + i] = cs[c][i] * a + sn[c][i] * b;
            Hc[(size_t)j * (m + 1) + i + 1] = -sn[c][i] * a + cs[c][i] * b;
          }
          const double a = Hc[(size_t)j * (m + 1) + j], b = Hc[(size_t)j * (m + 1) + j + 1];
          const double r = std::hypot(a, b);
          cs[c][j] = r > 0 ? a / r : 1.0;
          sn[c][j] = r > 0 ? b / r : 0.0;
          Hc[(size_t)j * (m + 1) + j] = r;
          Hc[(size_t)j * (m + 1) + j + 1] = 0.0;
          g[c][j + 1] = -sn[c][j] * g[c][j];
          g[c][j] = cs[c][j] * g[c][j];
          jc[c] = j + 1;
          if (std::fabs(g[c][j + 1]) <= 0.5 * tol * bn[c] || !(nrm[c] > 0.0)) conv[c] = 1;
          if (!conv[c]) all = false;
        }
        if (all) {
          ++j;
          break;
        }
      }
      // y from the triangular systems, X += M^-1 (V y)
      std::vector<double> y((size_t)m * q, 0.0);
      for (int c = 0; c < q; ++c) {
        for (int i = jc[c] - 1; i >= 0; --i) {
          double a = g[c][i];
          for (int k = i + 1; k < jc[c]; ++k) a -= H[c][(size_t)k * (m + 1) + i] * y[(size_t)k * q + c];
          const double d = H[c][(size_t)i * (m + 1) + i];
          y[(size_t)i * q + c] = d != 0.0 ? a / d : 0.0;
        }
      }
      hck(cudaMemcpyAsync(h, y.data(), sizeof(double) * m * q, cudaMemcpyHostToDevice, s), "GMRES solution");
      k_combine<<<gb, 256, 0, s>>>(n3, q, j, V, h, W, 0);
      BGPU_COUNT_LAUNCH();
      I.precond(q, W, n3, Z, n3, s);
      k_add<<<gb, 256, 0, s>>>(n3 * q, Z, X);
      BGPU_COUNT_LAUNCH();
      hck(cudaGetLastError(), "GMRES");
    }
    k_scatter_rows<<<gb, 256, 0, s>>>(I.n, I.perm.as<int>(), X, n3, q, d_b + (size_t)c0 * ldb, ldb);
    BGPU_COUNT_LAUNCH();
    hck(cudaStreamSynchronize(s), "GMRES");
    out.iterations = std::max(out.iterations, steps);
    out.restarts = std::max(out.restarts, restarts);
    out.relres = std::max(out.relres, worst);
  }
  I.last = out;
  if (rep) *rep = out;
}

std::vector<double> HMatrixSolver::stats() const {
  const Impl& I = *p_;
  return {(double)I.n,
          (double)I.leaves.size(),
          (double)I.dense.size(),
          (double)I.low.size(),
          I.dense_entries,
          I.low_entries,
          I.mean_rank,
          (double)I.max_rank,
          (double)I.capped,
          I.ms_fill,
          I.ms_aca,
          I.ms_pre,
          (double)I.last.iterations,
          I.last.relres,
          (double)I.held()};
}

}  // namespace bgpu
