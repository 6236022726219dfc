// Mixed-precision factorisation of BEST's GR and the refined solve (BF16 tensor cores + FP64
// GMRES iterative refinement).
//
// What it replaces: LAPACK dgetrf/dgetrs in FP64 (best/best.f:444, best/besolve.f90:133), or the
// H-matrix solver's GMRES behind bhm_build/bhm_solve (hmatrix/src/api.cpp:694-771), whose outer
// loop (several right-hand sides in lockstep, true residual at each restart) this follows.
//
// Factorisation: GR is assembled once in FP64 (kept for the residuals) with an FP32 copy written by
// the same kernel; the copy is factored without pivoting (as the reference's H-LU factors GR,
// hmatrix/src/hmatrix.cpp:1007) by recursive halving:
//     LU(D) = [L11 0; L21 L22][U11 U12; 0 U22]:  LU(D11); U12 = L11^-1 D12; L21 = D21 U11^-1;
//     D22 -= L21 U12; LU(D22)
// with 128 x 128 diagonal leaves factored in one CTA and inverted right away, triangular solves
// recursive down to 128-wide leaves that multiply by those inverses (FP32), and every other update
// C -= A B on the tcgen05 GEMM (BF16 operands, FP32 accumulation).
// Deflation keeps GR far from singular (1-norm condition ~1e3 on the synthetic meshes), so BF16
// updates are recovered by refinement in a few steps.
//
// Solve: restarted right-preconditioned GMRES in FP64 (preconditioner: the FP32 factors, applied
// entirely in FP32 -- vectors, partial sums and diagonal-block products; its result only steers the
// iteration), the true FP64 residual b - GR x at every restart; all right-hand sides
// advance in lockstep.  Stops at a relative residual of tol for every column; a failure to converge
// or a zero pivot is an error (the C ABI then factors the kept FP64 matrix instead).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "mixed.h"

namespace bgpu {
namespace {

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() {
    if (p) cudaFree(p);
  }
  void ensure(size_t need, const char* what) {
    if (p && bytes >= need) return;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (cudaMalloc(&p, need) != cudaSuccess) {
      cudaGetLastError();
      throw std::runtime_error(std::string("cannot allocate ") + what + " (" + std::to_string(need / 1e9) + " GB)");
    }
    bytes = need;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

constexpr int kLeaf = 128;
constexpr int kZeroPivot = 4;  // status: a pivot of the unpivoted FP32 LU is zero or not finite

long round_up(long v, long q) { return (v + q - 1) / q * q; }

// ---- diagonal leaf: h x h (h <= 128) LU without pivoting and the inverses of both triangles ----
// One CTA of 512 threads, everything in shared memory: M (the block, becoming L\U), LI = L^-1 and
// UI = U^-1, column-major with stride kS (rows and columns beyond h hold the identity, so the padded
// part factors to itself).  Recursive halving, as the factorisation around it:
//   LU(D) = [L11 0; L21 L22][U11 U12; 0 U22]:  LU(D11) with LI11, UI11;  U12 = LI11 D12 and
//   L21 = D21 UI11 (two thread groups at once);  D22 -= L21 U12;  LU(D22) with LI22, UI22;
//   LI21 = -LI22 (L21 LI11),  UI12 = -(UI11 U12) UI22  (the block inverse of a triangular matrix).
// 128 -> 64 -> 32; a 32 x 32 block is factored by one warp (lane i holds row i; row k of U goes to
// the other lanes by shuffles), and its two inverses by two warps (lane c forms column c by
// substitution).  Every product of the 64 and 128 levels is a small shared-memory matrix product
// with register tiles.  The serial part is 4 warp-sized factorisations; the rest is parallel.
constexpr int kS = 132;  // column stride (floats): 16-byte aligned columns

// Optional launch stamps (as the GEMM's): the earliest CTA start into st[0], the latest CTA end into
// st[1], global timer in ns.  st is a kernel argument, so the branch is uniform.
__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
  return t;
}
// (every kernel of the factorisation's chain starts here: the wait for its predecessor under
// programmatic dependent launch, the trigger for its successor, then the stamp)
__device__ __forceinline__ void stamp_begin(unsigned long long* st) {
  pdl_wait();
  pdl_trigger();
  if (st && threadIdx.x == 0) atomicMin(st, gtimer_ns());
}
__device__ __forceinline__ void stamp_end(unsigned long long* st) {
  if (st) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicMax(st + 1, gtimer_ns());
    }
  }
}

// group-local barrier (named barrier id, nthreads of the group)
__device__ __forceinline__ void group_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}

// C = A B (MODE 0), C = -A B (MODE 1), C -= A B (MODE 2) for H x H blocks (stride kS), by the NT
// threads t of a group.  C may alias A or B: every thread's products are finished (group barrier
// bar) before any is stored.  bar < 0: no aliasing, no barrier.
template <int H, int NT, int MODE>
__device__ __forceinline__ void small_mm(const float* A, const float* B, float* C, int t, int bar) {
  constexpr int OUT = H * H / NT;
  constexpr int TR = OUT >= 4 ? 4 : OUT;
  constexpr int TC = OUT / TR;
  constexpr int RG = H / TR;
  const int r0 = (t % RG) * TR, c0 = (t / RG) * TC;
  float acc[TR][TC];
#pragma unroll
  for (int i = 0; i < TR; ++i)
#pragma unroll
    for (int j = 0; j < TC; ++j) acc[i][j] = 0.f;
  // four k at a time: B's columns are contiguous in k (16-byte loads), A's in the row index
#pragma unroll 2
  for (int k = 0; k < H; k += 4) {
    float b[TC][4];
#pragma unroll
    for (int j = 0; j < TC; ++j) {
      const float4 v = *reinterpret_cast<const float4*>(B + (c0 + j) * kS + k);
      b[j][0] = v.x, b[j][1] = v.y, b[j][2] = v.z, b[j][3] = v.w;
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      float a[TR];
      if constexpr (TR == 4) {
        const float4 v = *reinterpret_cast<const float4*>(A + (k + kk) * kS + r0);
        a[0] = v.x, a[1] = v.y, a[2] = v.z, a[3] = v.w;
      } else {
#pragma unroll
        for (int i = 0; i < TR; ++i) a[i] = A[(k + kk) * kS + r0 + i];
      }
#pragma unroll
      for (int i = 0; i < TR; ++i)
#pragma unroll
        for (int j = 0; j < TC; ++j) acc[i][j] += a[i] * b[j][kk];
    }
  }
  if (bar >= 0) group_bar(bar, NT);
#pragma unroll
  for (int i = 0; i < TR; ++i)
#pragma unroll
    for (int j = 0; j < TC; ++j) {
      float* c = C + (c0 + j) * kS + r0 + i;
      if constexpr (MODE == 0) *c = acc[i][j];
      if constexpr (MODE == 1) *c = -acc[i][j];
      if constexpr (MODE == 2) *c -= acc[i][j];
    }
}

// One doubling step of a 32 x 32 triangular inverse by one warp (T the triangle, X its inverse, both
// at (o, o) of stride-kS column-major blocks): with the inverses of the S x S diagonal blocks of every
// 2S x 2S diagonal block already in X, the off-diagonal S x S block of each 2S block's inverse,
//   lower: X21 = -X22 (T21 X11),   upper: X12 = -X11 (T12 X22),
// the product in parentheses staged in X21 (X12) itself.  16 S outputs, S / 2 per lane (16 lanes for
// S = 1); each a full S-term sum (the zero triangles of X take part).
template <int S, bool LOWER>
__device__ __forceinline__ void tri_inv_step(const float* T, float* X, int o, int lane) {
  constexpr int NOUT = 16 * S, Q = NOUT >= 32 ? NOUT / 32 : 1;
  auto at = [o](int r, int c) { return (o + c) * kS + o + r; };
  float y[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int e = lane + 32 * q, p = e / (S * S), rem = e % (S * S), i = rem % S, j = rem / S, b = 2 * S * p;
    float acc = 0.f;
    if (e < NOUT) {
#pragma unroll
      for (int k = 0; k < S; ++k)
        acc += LOWER ? T[at(b + S + i, b + k)] * X[at(b + k, b + j)] : T[at(b + i, b + S + k)] * X[at(b + S + k, b + S + j)];
    }
    y[q] = acc;
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int e = lane + 32 * q, p = e / (S * S), rem = e % (S * S), i = rem % S, j = rem / S, b = 2 * S * p;
    if (e < NOUT) X[LOWER ? at(b + S + i, b + j) : at(b + i, b + S + j)] = y[q];
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int e = lane + 32 * q, p = e / (S * S), rem = e % (S * S), i = rem % S, j = rem / S, b = 2 * S * p;
    float acc = 0.f;
    if (e < NOUT) {
#pragma unroll
      for (int k = 0; k < S; ++k)
        acc += LOWER ? X[at(b + S + i, b + S + k)] * X[at(b + S + k, b + j)] : X[at(b + i, b + k)] * X[at(b + k, b + S + j)];
    }
    y[q] = -acc;
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int e = lane + 32 * q, p = e / (S * S), rem = e % (S * S), i = rem % S, j = rem / S, b = 2 * S * p;
    if (e < NOUT) X[LOWER ? at(b + S + i, b + j) : at(b + i, b + S + j)] = y[q];
  }
  __syncwarp();
}

// The inverse of the 32 x 32 triangle of T at (o, o) into X (zero there beforehand): lower with unit
// diagonal, or upper; five doubling steps from the diagonal up (log-depth, no 32-step substitution).
template <bool LOWER>
__device__ __forceinline__ void tri_inv32(const float* T, float* X, int o, int lane) {
  X[(o + lane) * kS + o + lane] = LOWER ? 1.f : 1.f / T[(o + lane) * kS + o + lane];
  __syncwarp();
  tri_inv_step<1, LOWER>(T, X, o, lane);
  tri_inv_step<2, LOWER>(T, X, o, lane);
  tri_inv_step<4, LOWER>(T, X, o, lane);
  tri_inv_step<8, LOWER>(T, X, o, lane);
  tri_inv_step<16, LOWER>(T, X, o, lane);
}

// The 32 x 32 diagonal block at (o, o): LU by warp 0, then L^-1 by warp 0 and U^-1 by warp 1.
// Called by all threads (it ends with a block barrier).
__device__ __noinline__ void leaf_base32(float* M, float* LI, float* UI, int o, int* bad) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    float r[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = M[(o + j) * kS + o + lane];
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const float ukk = __shfl_sync(0xffffffffu, r[k], k);
      if (lane == 0 && !(ukk != 0.f && isfinite(ukk))) *bad = 1;
      const float l = r[k] * (1.0f / ukk);
      if (lane > k) r[k] = l;
#pragma unroll
      for (int j = k + 1; j < 32; ++j) {
        const float ukj = __shfl_sync(0xffffffffu, r[j], k);
        if (lane > k) r[j] -= l * ukj;
      }
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) M[(o + j) * kS + o + lane] = r[j];
  }
  __syncthreads();
  if (warp == 0)
    tri_inv32<true>(M, LI, o, lane);
  else if (warp == 1)
    tri_inv32<false>(M, UI, o, lane);
  __syncthreads();
}

// One level of the recursion: the H x H diagonal block at (o, o) from its two halves (h = H / 2).
// Thread groups: warps 0-7 (id 1) and 8-15 (id 2), 256 threads each.
template <int H>
__device__ __forceinline__ void leaf_level(float* M, float* LI, float* UI, int o, int* bad) {
  constexpr int h = H / 2;
  if constexpr (h == 32) {
    leaf_base32(M, LI, UI, o, bad);
  } else {
    leaf_level<h>(M, LI, UI, o, bad);
  }
  const int tid = threadIdx.x, grp = tid >> 8, t = tid & 255;
  const int p = o + h;  // second half
  float* M11 = M + o * kS + o;
  float* M12 = M + p * kS + o;
  float* M21 = M + o * kS + p;
  float* M22 = M + p * kS + p;
  // U12 = LI11 D12 (group 1), L21 = D21 UI11 (group 2), in place
  if (grp == 0)
    small_mm<h, 256, 0>(LI + o * kS + o, M12, M12, t, 1);
  else
    small_mm<h, 256, 0>(M21, UI + o * kS + o, M21, t, 2);
  __syncthreads();
  small_mm<h, 512, 2>(M21, M12, M22, tid, -1);  // D22 -= L21 U12
  __syncthreads();
  if constexpr (h == 32) {
    leaf_base32(M, LI, UI, p, bad);
  } else {
    leaf_level<h>(M, LI, UI, p, bad);
  }
  // LI21 = -LI22 (L21 LI11) (group 1), UI12 = -(UI11 U12) UI22 (group 2)
  float* LI21 = LI + o * kS + p;
  float* UI12 = UI + p * kS + o;
  if (grp == 0) {
    small_mm<h, 256, 0>(M21, LI + o * kS + o, LI21, t, -1);
    group_bar(1, 256);
    small_mm<h, 256, 1>(LI + p * kS + p, LI21, LI21, t, 1);
  } else {
    small_mm<h, 256, 0>(UI + o * kS + o, M12, UI12, t, -1);
    group_bar(2, 256);
    small_mm<h, 256, 1>(UI12, UI + p * kS + p, UI12, t, 2);
  }
  __syncthreads();
  (void)M11;
}

__global__ void __launch_bounds__(512, 1) k_lu32_leaf_inv(float* __restrict__ A, long lda, int h, float* __restrict__ DL,
                                                           float* __restrict__ DU, int* status,
                                                           unsigned long long* stamp) {
  stamp_begin(stamp);
  extern __shared__ __align__(16) float sm[];
  float* M = sm;
  float* LI = sm + 128 * kS;
  float* UI = sm + 2 * 128 * kS;
  __shared__ int s_bad;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) s_bad = 0;
  if (h == 128) {
    float4 v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = *reinterpret_cast<const float4*>(A + (size_t)(warp + 16 * q) * lda + 4 * lane);
#pragma unroll
    for (int q = 0; q < 8; ++q) *reinterpret_cast<float4*>(M + (warp + 16 * q) * kS + 4 * lane) = v[q];
  } else {
    for (int c = warp; c < 128; c += 16)
      for (int r = lane; r < 128; r += 32)
        M[c * kS + r] = (r < h && c < h) ? A[(size_t)c * lda + r] : (r == c ? 1.f : 0.f);
  }
  // LI and UI start at zero (the blocks above / below their diagonals stay zero)
  for (int e = tid; e < 2 * 128 * kS / 4; e += 512) reinterpret_cast<float4*>(LI)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  leaf_level<128>(M, LI, UI, 0, &s_bad);
  if (h == 128) {
#pragma unroll
    for (int q = 0; q < 8; ++q)
      *reinterpret_cast<float4*>(A + (size_t)(warp + 16 * q) * lda + 4 * lane) =
          *reinterpret_cast<const float4*>(M + (warp + 16 * q) * kS + 4 * lane);
  } else {
    for (int c = warp; c < h; c += 16)
      for (int r = lane; r < h; r += 32) A[(size_t)c * lda + r] = M[c * kS + r];
  }
  // L^-1 and U^-1, 128 x 128 column-major, zero outside h x h
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int c = warp + 16 * q, r = 4 * lane;
    float4 l = *reinterpret_cast<const float4*>(LI + c * kS + r);
    float4 u = *reinterpret_cast<const float4*>(UI + c * kS + r);
    if (h < 128) {
      const bool cin = c < h;
      l.x = (cin && r < h) ? l.x : 0.f, l.y = (cin && r + 1 < h) ? l.y : 0.f;
      l.z = (cin && r + 2 < h) ? l.z : 0.f, l.w = (cin && r + 3 < h) ? l.w : 0.f;
      u.x = (cin && r < h) ? u.x : 0.f, u.y = (cin && r + 1 < h) ? u.y : 0.f;
      u.z = (cin && r + 2 < h) ? u.z : 0.f, u.w = (cin && r + 3 < h) ? u.w : 0.f;
    }
    *reinterpret_cast<float4*>(DL + (size_t)c * 128 + r) = l;
    *reinterpret_cast<float4*>(DU + (size_t)c * 128 + r) = u;
  }
  __syncthreads();
  if (tid == 0 && s_bad) atomicExch(status, kZeroPivot);
  stamp_end(stamp);
}

// 16-byte asynchronous copy global -> shared; fewer than 16 source bytes are zero-filled
__device__ __forceinline__ void cp16(void* sdst, const void* gsrc, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The inverse of the 256 x 256 diagonal block at (k0, k0) from its two 128-block inverses, for the
// 256-deep triangular-solve leaves (k_leaf256_tf32), column-major 256 x 256 into T:
//   lower (blockIdx.y == 0): [[D1, 0], [F, D2]],  F = -D2 (L21 D1),  D = the unit-lower inverses (DL)
//   upper (blockIdx.y == 1): [[E1, G], [0, E2]],  G = -E1 (U12 E2),  E = the upper inverses (DU)
// L21 = the factor's block (k0 + 128, k0), U12 = (k0, k0 + 128).  CTA x: columns 16 x .. 16 x + 15
// of each 128-column half; FP32 CUDA cores (two 128 x 128 x 16 products per CTA).
constexpr size_t kCombineSmem = (size_t)(128 * 129 + 2 * 128 * 16) * sizeof(float);
__global__ void __launch_bounds__(256) k_combine256(const float* __restrict__ LU, long lda, int k0,
                                                     const float* __restrict__ DL, const float* __restrict__ DU,
                                                     float* __restrict__ TL, float* __restrict__ TU,
                                                     unsigned long long* stamp) {
  stamp_begin(stamp);
  extern __shared__ __align__(16) float sm[];
  float* sA = sm;                     // a 128 x 128 operand, (r, k) at sA[k * 129 + r]
  float* sB = sm + 128 * 129;         // the 128 x 16 slab operand, (k, c) at sB[k * 16 + c]
  float* sT = sB + 128 * 16;          // the 128 x 16 intermediate
  const bool lower = blockIdx.y == 0;
  const int c0 = 16 * blockIdx.x, tid = threadIdx.x, r = tid & 127, ch = (tid >> 7) * 8;
  const int b = k0 / 128;
  const float* X1 = (lower ? DL : DU) + (size_t)b * 16384;        // D1 or E1
  const float* X2 = (lower ? DL : DU) + (size_t)(b + 1) * 16384;  // D2 or E2
  const float* off = lower ? LU + (size_t)k0 * lda + k0 + 128 : LU + (size_t)(k0 + 128) * lda + k0;  // L21 or U12
  float* T = (lower ? TL : TU) + (size_t)b * 65536;
  // a 128 x 128 column-major block (leading dimension ld, 16-byte aligned columns) into sA: sixteen
  // 16-byte loads in flight per thread
  auto stage = [&](const float* src, long ld) {
    float4 v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e4 = tid + 256 * q, col = e4 >> 5, row = (e4 & 31) * 4;
      v[q] = __ldg(reinterpret_cast<const float4*>(src + (size_t)col * ld + row));
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e4 = tid + 256 * q, col = e4 >> 5, row = (e4 & 31) * 4;
      float* d = sA + col * 129 + row;
      d[0] = v[q].x, d[1] = v[q].y, d[2] = v[q].z, d[3] = v[q].w;
    }
  };
  // product 1: lower L21 D1[:, slab], upper U12 E2[:, slab]
  stage(off, lda);
  const float* s1 = lower ? X1 : X2;
  {
    float b8[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + 256 * q;
      b8[q] = __ldg(s1 + (size_t)(c0 + (e >> 7)) * 128 + (e & 127));
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + 256 * q;
      sB[(e & 127) * 16 + (e >> 7)] = b8[q];
    }
  }
  __syncthreads();
  float acc[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) acc[c] = 0.f;
  for (int k = 0; k < 128; ++k) {
    const float a = sA[k * 129 + r];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] += a * sB[k * 16 + ch + c];
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) sT[r * 16 + ch + c] = acc[c];
  __syncthreads();
  // product 2: lower -D2 T, upper -E1 T
  stage(lower ? X2 : X1, 128);
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 8; ++c) acc[c] = 0.f;
  for (int k = 0; k < 128; ++k) {
    const float a = sA[k * 129 + r];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] += a * sT[k * 16 + ch + c];
  }
  // columns c0 + c of the left half and 128 + c0 + c of the right half, all 256 rows (the copies of
  // D1, D2 / E1, E2 loaded before any store)
  float x1[8], x2[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int j = c0 + ch + c;
    x1[c] = __ldg(X1 + (size_t)j * 128 + r);
    x2[c] = __ldg(X2 + (size_t)j * 128 + r);
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int j = c0 + ch + c;
    float* left = T + (size_t)j * 256;
    float* right = T + (size_t)(128 + j) * 256;
    left[r] = x1[c];
    left[128 + r] = lower ? -acc[c] : 0.f;
    right[r] = lower ? 0.f : -acc[c];
    right[128 + r] = x2[c];
  }
  stamp_end(stamp);
}

constexpr int kLm = 132;  // row stride of the shared operands (floats)
constexpr int kWideLeaf = 8192;  // from this many columns (rows) on, k_leaf_mult; below, 64 per CTA
template <bool LEFT>
__global__ void __launch_bounds__(256, 1) k_leaf_mult(const float* __restrict__ Dinv, int h, float* B, long ldb,
                                                      int len, __nv_bfloat16* __restrict__ mir, long ldm,
                                                      unsigned long long* stamp) {
  stamp_begin(stamp);
  extern __shared__ __align__(16) float sm[];
  float* As = sm;               // As[k * kLm + i]: the left factor's (i, k)
  float* Bs = sm + 128 * kLm;   // Bs[k * kLm + j]: the right factor's (k, j)
  const int tid = threadIdx.x;
  const int t0 = blockIdx.x * 128, nt = min(128, len - t0);  // this CTA's columns (LEFT) or rows of B
  // operands in: rows of shared memory that are contiguous in global memory by 16-byte asynchronous
  // copies, transposed ones by float4 loads (all issued before any is used)
  const float* tsrc;  // the operand stored transposed: element (k, x) at tsrc[x * tld + k]
  long tld;
  int tk, tx_lim;     // its valid k and x ranges
  float* tdst;
  if (LEFT) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {  // Dinv column k -> As row k
      const int e = tid + 256 * q, k = e >> 5, i4 = (e & 31) * 4;
      cp16(&As[k * kLm + i4], &Dinv[(size_t)k * 128 + i4], 16);
    }
    tsrc = B + (size_t)t0 * ldb;  // B (k, t0 + j) at B[(t0 + j) ldb + k]
    tld = ldb;
    tk = h;
    tx_lim = nt;
    tdst = Bs;
  } else {
#pragma unroll
    for (int q = 0; q < 16; ++q) {  // B (t0 + i, k), i contiguous -> As row k
      const int e = tid + 256 * q, k = e >> 5, i4 = (e & 31) * 4;
      const int valid = (k < h) ? max(0, min(4, nt - i4)) * 4 : 0;
      cp16(&As[k * kLm + i4], valid ? (const void*)&B[(size_t)k * ldb + t0 + i4] : (const void*)B, valid);
    }
    tsrc = Dinv;  // Dinv (k, j) at Dinv[j * 128 + k]
    tld = 128;
    tk = 128;
    tx_lim = 128;
    tdst = Bs;
  }
  {
    // lanes along x: the transposed stores of a warp hit 32 consecutive words (no bank conflicts)
    float4 v[16];
    const int x = tid & 127;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int k4 = ((tid >> 7) + 2 * q) * 4;
      v[q] = (x < tx_lim && k4 < tk) ? *reinterpret_cast<const float4*>(&tsrc[(size_t)x * tld + k4])
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int k4 = ((tid >> 7) + 2 * q) * 4;
      tdst[(k4 + 0) * kLm + x] = k4 + 0 < tk ? v[q].x : 0.f;
      tdst[(k4 + 1) * kLm + x] = k4 + 1 < tk ? v[q].y : 0.f;
      tdst[(k4 + 2) * kLm + x] = k4 + 2 < tk ? v[q].z : 0.f;
      tdst[(k4 + 3) * kLm + x] = k4 + 3 < tk ? v[q].w : 0.f;
    }
  }
  cp_wait_all();
  __syncthreads();
  const int ty = tid >> 4, tx = tid & 15;  // rows 8 ty .. +7, columns 4 tx .. +3 and 64 + 4 tx .. +3
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
#pragma unroll 4
  for (int k = 0; k < 128; ++k) {
    const float4 a0 = *reinterpret_cast<const float4*>(&As[k * kLm + 8 * ty]);
    const float4 a1 = *reinterpret_cast<const float4*>(&As[k * kLm + 8 * ty + 4]);
    const float4 b0 = *reinterpret_cast<const float4*>(&Bs[k * kLm + 4 * tx]);
    const float4 b1 = *reinterpret_cast<const float4*>(&Bs[k * kLm + 64 + 4 * tx]);
    const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] += av[i] * bv[j];
  }
  // results through shared memory (Cs[jj * kLm + ii]: local row ii, local column jj of B's block),
  // then coalesced stores
  __syncthreads();
  float* Cs = sm;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int jj = j < 4 ? 4 * tx + j : 64 + 4 * tx + (j - 4);
#pragma unroll
    for (int i = 0; i < 8; ++i) Cs[jj * kLm + 8 * ty + i] = acc[i][j];
  }
  __syncthreads();
  if (LEFT) {
    // B rows ii < h, columns t0 + jj (jj < nt); mirror column-major
    for (int e = tid; e < 128 * 128; e += 256) {
      const int ii = e & 127, jj = e >> 7;
      if (ii < h && jj < nt) {
        const float v = Cs[jj * kLm + ii];
        B[(size_t)(t0 + jj) * ldb + ii] = v;
        if (mir) mir[(size_t)(t0 + jj) * ldm + ii] = __float2bfloat16_rn(v);
      }
    }
  } else {
    // B rows t0 + ii (ii < nt), columns jj < h; mirror row-major
    for (int e = tid; e < 128 * 128; e += 256) {
      const int ii = e & 127, jj = e >> 7;
      if (ii < nt && jj < h) B[(size_t)jj * ldb + t0 + ii] = Cs[jj * kLm + ii];
    }
    if (mir)
      for (int e = tid; e < 128 * 128; e += 256) {
        const int jj = e & 127, ii = e >> 7;
        if (ii < nt && jj < h) mir[(size_t)(t0 + ii) * ldm + jj] = __float2bfloat16_rn(Cs[jj * kLm + ii]);
      }
  }
  stamp_end(stamp);
}

// The narrow leaves (fewer than kWideLeaf columns or rows), FP32, 256 threads, NB = 64, 32 or 16
// columns (rows) of B per CTA, each thread 4 rows x NB/8 columns of the result; the narrower
// the leaf, the fewer per CTA, so that the grid still covers every SM.  Mirror writes as
// k_leaf_mult's.
constexpr int kLdI = 132;
template <int NB>
struct NarrowLeaf {
  static constexpr int kCpt = NB / 8;    // result columns per thread
  static constexpr int kLdB = NB + 4;    // row stride of the staged B block (floats)
  static constexpr size_t smem() { return (size_t)(128 * kLdI + 128 * kLdB) * sizeof(float); }
};

// kCpt consecutive floats of shared memory (kCpt = 8, 4 or 2; 8-byte aligned at least)
template <int C>
__device__ __forceinline__ void lds_n(const float* p, float (&v)[C]) {
  if constexpr (C == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    v[0] = t.x, v[1] = t.y;
  } else {
#pragma unroll
    for (int q = 0; q < C / 4; ++q) {
      const float4 t = *reinterpret_cast<const float4*>(p + 4 * q);
      v[4 * q] = t.x, v[4 * q + 1] = t.y, v[4 * q + 2] = t.z, v[4 * q + 3] = t.w;
    }
  }
}

// B (h x w, ldb) := Dinv B, Dinv an inverse diagonal block (128 x 128, ld 128, zero outside h)
template <int NB>
__global__ void __launch_bounds__(256) k_apply_inv_left(const float* __restrict__ Dinv, int h, float* B, long ldb,
                                                         int w, __nv_bfloat16* __restrict__ mir, long ldm,
                                                         unsigned long long* stamp) {
  stamp_begin(stamp);
  using L = NarrowLeaf<NB>;
  constexpr int C = L::kCpt, ldb_s = L::kLdB;
  extern __shared__ __align__(16) float sm[];
  float* li = sm;                 // li[k * kLdI + r] = Dinv(r, k)
  float* bs = sm + 128 * kLdI;    // bs[k * ldb_s + c] = B(k, c0 + c)
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * NB, nc = min(NB, w - c0);
#pragma unroll
  for (int q = 0; q < 16; ++q) {  // Dinv column k -> li row k (16-byte asynchronous copies)
    const int e = tid + 256 * q, k = e >> 5, r4 = (e & 31) * 4;
    cp16(&li[k * kLdI + r4], &Dinv[(size_t)k * 128 + r4], 16);
  }
  {
    // B (k, c0 + cc), k contiguous in memory: float4 loads, transposed into bs with the lanes along
    // cc (no bank conflicts on the stores)
    float4 v[NB / 8];
#pragma unroll
    for (int q = 0; q < NB / 8; ++q) {
      const int e = tid + 256 * q, cc = e % NB, k4 = (e / NB) * 4;
      v[q] = (cc < nc && k4 < h) ? *reinterpret_cast<const float4*>(&B[(size_t)(c0 + cc) * ldb + k4])
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < NB / 8; ++q) {
      const int e = tid + 256 * q, cc = e % NB, k4 = (e / NB) * 4;
      bs[(k4 + 0) * ldb_s + cc] = k4 + 0 < h ? v[q].x : 0.f;
      bs[(k4 + 1) * ldb_s + cc] = k4 + 1 < h ? v[q].y : 0.f;
      bs[(k4 + 2) * ldb_s + cc] = k4 + 2 < h ? v[q].z : 0.f;
      bs[(k4 + 3) * ldb_s + cc] = k4 + 3 < h ? v[q].w : 0.f;
    }
  }
  cp_wait_all();
  __syncthreads();
  const int tr = tid & 31, tc = tid >> 5;  // rows 4 tr .. 4 tr + 3, columns C tc .. C tc + C - 1
  float acc[4][C];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < C; ++j) acc[i][j] = 0.f;
  for (int k = 0; k < h; ++k) {
    const float4 a = *reinterpret_cast<const float4*>(&li[k * kLdI + 4 * tr]);
    float bv[C];
    lds_n<C>(&bs[k * ldb_s + C * tc], bv);
    const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < C; ++j) acc[i][j] += av[i] * bv[j];
  }
#pragma unroll
  for (int j = 0; j < C; ++j) {
    const int cc = C * tc + j;
    if (cc < nc)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = 4 * tr + i;
        if (r < h) {
          B[(size_t)(c0 + cc) * ldb + r] = acc[i][j];
          if (mir) mir[(size_t)(c0 + cc) * ldm + r] = __float2bfloat16_rn(acc[i][j]);
        }
      }
  }
  stamp_end(stamp);
}

// B (m x h, ldb) := B Dinv, Dinv an inverse diagonal block (128 x 128, ld 128, zero outside h)
template <int NB>
__global__ void __launch_bounds__(256) k_apply_inv_right(const float* __restrict__ Dinv, int h, float* B, long ldb,
                                                          int m, __nv_bfloat16* __restrict__ mir, long ldm,
                                                          unsigned long long* stamp) {
  stamp_begin(stamp);
  using L = NarrowLeaf<NB>;
  constexpr int C = L::kCpt, ldb_s = L::kLdB, RG = NB / 4;  // RG row groups of 4
  extern __shared__ __align__(16) float sm[];
  float* us = sm;                 // us[k * kLdI + c] = Dinv(k, c)
  float* bs = sm + 128 * kLdI;    // bs[k * ldb_s + rr] = B(r0 + rr, k)
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * NB, nr = min(NB, m - r0);
#pragma unroll
  for (int q = 0; q < NB / 8; ++q) {  // B (r0 + rr, k), rr contiguous -> bs row k (16-byte copies)
    const int e = tid + 256 * q, k = e / RG, rr4 = (e % RG) * 4;
    const int valid = (k < h) ? max(0, min(4, nr - rr4)) * 4 : 0;
    cp16(&bs[k * ldb_s + rr4], valid ? (const void*)&B[(size_t)k * ldb + r0 + rr4] : (const void*)B, valid);
  }
  {
    // Dinv (k, cc) at Dinv[cc * 128 + k]: float4 loads along k, transposed into us with the lanes
    // along cc (no bank conflicts on the stores)
    float4 v[16];
    const int cc = tid & 127;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int k4 = ((tid >> 7) + 2 * q) * 4;
      v[q] = *reinterpret_cast<const float4*>(&Dinv[(size_t)cc * 128 + k4]);
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int k4 = ((tid >> 7) + 2 * q) * 4;
      us[(k4 + 0) * kLdI + cc] = v[q].x;
      us[(k4 + 1) * kLdI + cc] = v[q].y;
      us[(k4 + 2) * kLdI + cc] = v[q].z;
      us[(k4 + 3) * kLdI + cc] = v[q].w;
    }
  }
  cp_wait_all();
  __syncthreads();
  const int tr = tid % RG, tc = tid / RG;  // rows 4 tr .. 4 tr + 3, columns C tc .. C tc + C - 1
  float acc[4][C];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < C; ++j) acc[i][j] = 0.f;
  for (int k = 0; k < h; ++k) {
    const float4 a = *reinterpret_cast<const float4*>(&bs[k * ldb_s + 4 * tr]);
    float bv[C];
    lds_n<C>(&us[k * kLdI + C * tc], bv);
    const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < C; ++j) acc[i][j] += av[i] * bv[j];
  }
#pragma unroll
  for (int j = 0; j < C; ++j) {
    const int cc = C * tc + j;
    if (cc < h)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rr = 4 * tr + i;
        if (rr < nr) B[(size_t)cc * ldb + r0 + rr] = acc[i][j];
      }
  }
  if (mir) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int rr = 4 * tr + i;
      if (rr >= nr) continue;
      __nv_bfloat16* dst = mir + (size_t)(r0 + rr) * ldm + C * tc;
#pragma unroll
      for (int j = 0; j < C; ++j)
        if (C * tc + j < h) dst[j] = __float2bfloat16_rn(acc[i][j]);
    }
  }
  stamp_end(stamp);
}

// one narrow leaf: the per-CTA width that gives at least two CTAs per SM where it can
template <bool LEFT>
void launch_narrow_leaf(const float* dinv, int h, float* B, long ldb, int len, __nv_bfloat16* mir, long ldm,
                        int sms, cudaStream_t s, unsigned long long* st) {
  const int nb = len <= 2 * sms * 16 ? 16 : len <= 2 * sms * 32 ? 32 : 64;
#define BGPU_NARROW(NB)                                                                                  \
  if (LEFT)                                                                                              \
    launch_dependent(k_apply_inv_left<NB>, dim3((len + NB - 1) / NB), dim3(256), NarrowLeaf<NB>::smem(), s, dinv, h, \
                     B, ldb, len, mir, ldm, st);                                                         \
  else                                                                                                   \
    launch_dependent(k_apply_inv_right<NB>, dim3((len + NB - 1) / NB), dim3(256), NarrowLeaf<NB>::smem(), s, dinv, \
                     h, B, ldb, len, mir, ldm, st)
  if (nb == 16) {
    BGPU_NARROW(16);
  } else if (nb == 32) {
    BGPU_NARROW(32);
  } else {
    BGPU_NARROW(64);
  }
#undef BGPU_NARROW
}

// ---- small updates C -= A B in FP32 on the CUDA cores ------------------------------------------
// The recursion's smallest products (K <= 256, at most 2^26 multiply-adds, e.g. 128 x 128 x 128 or
// 1024 x 256 x 256) take 15-20 us each on the persistent tcgen05 kernel, whose start-up (TMEM
// allocation, barrier set-up, the first TMA round trip) is most of it; here 64 x 64 tiles, one per
// CTA, 4 x 4 results per thread, K in steps of 32 through shared memory.  FP32 operands straight
// from the factor (more accurate than the BF16 mirrors the tensor cores read).
constexpr int kSgBk = 32;
inline bool small_update(int m, int n, int k) { return k <= 256 && (long long)m * n * k <= (1LL << 26); }
// the K = 128 products of the TF32 panel kernel
inline bool panel_update(int m, int n, int k) {
  return k == 128 && (std::min(m, n) <= 128 || (std::min(m, n) <= 256 && std::max(m, n) <= 3840));
}
__global__ void __launch_bounds__(256) k_sgemm_small_minus(int m, int n, int k, const float* __restrict__ A, long lda,
                                                          const float* __restrict__ B, long ldb, float* __restrict__ C,
                                                          long ldc, unsigned long long* stamp) {
  stamp_begin(stamp);
  __shared__ __align__(16) float As[kSgBk][64 + 4];  // As[kk][r] = A(m0 + r, k0 + kk)
  __shared__ __align__(16) float Bs[kSgBk][64 + 4];  // Bs[kk][c] = B(k0 + kk, n0 + c)
  const int tid = threadIdx.x, tr = tid & 15, tc = tid >> 4;
  const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < k; k0 += kSgBk) {
    for (int e = tid; e < kSgBk * 64; e += 256) {
      const int kk = e >> 6, r = e & 63;
      As[kk][r] = (m0 + r < m && k0 + kk < k) ? A[(size_t)(k0 + kk) * lda + m0 + r] : 0.f;
    }
    for (int e = tid; e < kSgBk * 64; e += 256) {
      const int kk = e & (kSgBk - 1), c = e / kSgBk;
      Bs[kk][c] = (n0 + c < n && k0 + kk < k) ? B[(size_t)(n0 + c) * ldb + k0 + kk] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kSgBk; ++kk) {
      const float4 a = *reinterpret_cast<const float4*>(&As[kk][4 * tr]);
      const float4 b = *reinterpret_cast<const float4*>(&Bs[kk][4 * tc]);
      const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += av[i] * bv[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = n0 + 4 * tc + j;
    if (c >= n) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = m0 + 4 * tr + i;
      if (r < m) C[(size_t)c * ldc + r] -= acc[i][j];
    }
  }
  stamp_end(stamp);
}

// ---- FP64 mat-vec for the residuals: Y = beta Y + alpha A X (q <= Q columns) ----------------
// Four rows per thread (two 16-byte loads per column; the leading dimension is a multiple of 32 and
// the rows start at multiples of 4), the columns split over blockIdx.y into partial sums P, reduced
// in a fixed order afterwards.  X's chunk of kMvCols columns is staged in shared memory, and the
// loads of A go four columns ahead through the non-allocating streaming path: GR is read once per
// product and never reused, so it should not displace anything in L1.  (Measured on B200 at order
// 61,440, 6 right-hand sides: 4.81 ms, 6.28 TB/s, against 6.79 ms for two rows per thread with X
// read through L1.)
constexpr int kMvCols = 128;
__device__ __forceinline__ double2 ld_stream_f64x2(const double* p) {
  double2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
template <int Q>
__global__ void __launch_bounds__(128) k_matvec64_part(const double* __restrict__ A, long lda, int n,
                                                       const double* __restrict__ X, long ldx, int q, int cols_per,
                                                       double* __restrict__ P) {
  __shared__ double xs[kMvCols][Q];
  const int row = 4 * (blockIdx.x * 128 + threadIdx.x), split = blockIdx.y;
  const int c0 = split * cols_per, c1 = min(n, c0 + cols_per);
  double acc[4][Q];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < Q; ++j) acc[i][j] = 0.0;
  const bool live = row < n;
  const double* a = A + (live ? row : 0);
  for (int cb = c0; cb < c1; cb += kMvCols) {
    const int nc = min(kMvCols, c1 - cb);
    __syncthreads();
    for (int e = threadIdx.x; e < kMvCols * Q; e += 128) {
      const int c = e / Q, j = e % Q;
      xs[c][j] = (c < nc && j < q) ? X[(size_t)j * ldx + cb + c] : 0.0;
    }
    __syncthreads();
    if (live) {
      int c = 0;
      for (; c + 4 <= nc; c += 4) {
        double2 v[4][2];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          v[u][0] = ld_stream_f64x2(a + (size_t)(cb + c + u) * lda);
          v[u][1] = ld_stream_f64x2(a + (size_t)(cb + c + u) * lda + 2);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int j = 0; j < Q; ++j) {
            const double x = xs[c + u][j];
            acc[0][j] += v[u][0].x * x;
            acc[1][j] += v[u][0].y * x;
            acc[2][j] += v[u][1].x * x;
            acc[3][j] += v[u][1].y * x;
          }
      }
      for (; c < nc; ++c) {
        const double2 w0 = ld_stream_f64x2(a + (size_t)(cb + c) * lda);
        const double2 w1 = ld_stream_f64x2(a + (size_t)(cb + c) * lda + 2);
#pragma unroll
        for (int j = 0; j < Q; ++j) {
          const double x = xs[c][j];
          acc[0][j] += w0.x * x;
          acc[1][j] += w0.y * x;
          acc[2][j] += w1.x * x;
          acc[3][j] += w1.y * x;
        }
      }
    }
  }
  if (live) {
#pragma unroll
    for (int j = 0; j < Q; ++j)
      if (j < q)
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (row + i < n) P[((size_t)split * Q + j) * n + row + i] = acc[i][j];
  }
}

template <int Q>
__global__ void k_matvec64_reduce(const double* __restrict__ P, int n, int q, int splits, double alpha, double beta,
                                  double* Y, long ldy) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  for (int j = 0; j < q; ++j) {
    double s = 0.0;
    for (int t = 0; t < splits; ++t) s += P[((size_t)t * Q + j) * n + row];
    double* y = Y + (size_t)j * ldy + row;
    *y = (beta == 0.0 ? 0.0 : beta * *y) + alpha * s;
  }
}

// ---- small vector kernels for GMRES (all blocks of q columns, column c at c * n) ------------
// out[i * q + c] partial sums over a chunk of rows of V_i[c] . W[c], i < nv
__global__ void k_dots(const double* __restrict__ V, int nv, const double* __restrict__ W, int n, int q,
                       double* __restrict__ part) {
  const int i = blockIdx.y;
  __shared__ double red[16][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc[16];
  for (int c = 0; c < 16; ++c) acc[c] = 0.0;
  const double* v = V + (size_t)i * q * n;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int c = 0; c < q; ++c) acc[c] += v[(size_t)c * n + r] * W[(size_t)c * n + r];
  for (int c = 0; c < q; ++c) {
    double x = acc[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[c][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < q) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
    part[((size_t)blockIdx.x * nv + i) * q + threadIdx.x] = s;
  }
}

__global__ void k_dots_reduce(const double* __restrict__ part, int nparts, int count, double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  double s = 0.0;
  for (int p = 0; p < nparts; ++p) s += part[(size_t)p * count + t];
  out[t] = s;
}

// W[c] += sign * sum_i V_i[c] coef[i * q + c]
__global__ void k_combine(const double* __restrict__ V, int nv, const double* __restrict__ coef, double sign, double* W,
                          int n, int q) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int c = 0; c < q; ++c) {
      double s = 0.0;
      for (int i = 0; i < nv; ++i) s += V[((size_t)i * q + c) * n + r] * coef[i * q + c];
      W[(size_t)c * n + r] += sign * s;
    }
}

// Y[c] = X[c] * scale[c]
__global__ void k_scale_cols(const double* __restrict__ X, const double* __restrict__ scale, double* Y, int n, int q) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int c = 0; c < q; ++c) Y[(size_t)c * n + r] = X[(size_t)c * n + r] * scale[c];
}

// the preconditioner's FP32 copy of n x q FP64 vectors (ld n both), and back
__global__ void k_to_f32(const double* __restrict__ X, size_t len, float* __restrict__ Y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x)
    Y[i] = (float)X[i];
}
__global__ void k_to_f64(const float* __restrict__ X, size_t len, double* __restrict__ Y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x)
    Y[i] = (double)X[i];
}

__global__ void k_copy_in(const double* __restrict__ B, long ldb, int n, int q, double* Y) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int c = 0; c < q; ++c) Y[(size_t)c * n + r] = B[(size_t)c * ldb + r];
}
__global__ void k_copy_out(const double* __restrict__ Y, int n, int q, double* B, long ldb) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int c = 0; c < q; ++c) B[(size_t)c * ldb + r] = Y[(size_t)c * n + r];
}

// Optional per-call timing (BEST_GPU_PROFILE=1): CUDA events around each GEMM, cast and leaf,
// summed per category and (for GEMMs) per size class, reported as log lines after the build.
struct CallProfile {
  bool on = false;
  struct Rec {
    std::string key;
    cudaEvent_t a, b;
    double flops;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  cudaEvent_t ev() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  void begin(const std::string& key, double flops, cudaStream_t s) {
    if (!on) return;
    Rec r{key, ev(), ev(), flops};
    cudaEventRecord(r.a, s);
    recs.push_back(r);
  }
  void end(cudaStream_t s) {
    if (on) cudaEventRecord(recs.back().b, s);
  }
  std::vector<std::string> report() {
    std::vector<std::string> out;
    if (!on || recs.empty()) return out;
    cudaEventSynchronize(recs.back().b);
    std::map<std::string, std::pair<int, std::pair<double, double>>> agg;
    for (auto& r : recs) {
      float ms = 0;
      cudaEventElapsedTime(&ms, r.a, r.b);
      auto& a = agg[r.key];
      a.first += 1;
      a.second.first += ms;
      a.second.second += r.flops;
    }
    for (auto& kv : agg) {
      char buf[256];
      std::snprintf(buf, sizeof buf, "profile: %-28s %6d calls %9.2f ms %8.1f TFLOP/s", kv.first.c_str(),
                    kv.second.first, kv.second.second.first,
                    kv.second.second.second / std::max(1e-9, kv.second.second.first * 1e-3) / 1e12);
      out.emplace_back(buf);
    }
    recs.clear();
    used = 0;
    return out;
  }
};

// kinds of the factorisation's stamped launches
constexpr unsigned char kSlotGemm = 0, kSlotLuLeaf = 1, kSlotSolveLeaf = 2, kSlotSmall = 3, kSlotPanel = 4;

// The factorisation's timeline from its launch stamps, between the first start and the last end:
// how long a BF16 GEMM ran, else a TF32 panel update, else a small FP32 update, else only leaves
// (LU leaves among them), and how long nothing ran.
std::string timeline_note(const std::vector<unsigned long long>& h, const std::vector<unsigned char>& kind, int n) {
  std::vector<std::pair<unsigned long long, int>> ev;  // (time, +-(1 + kind))
  for (int i = 0; i < n; ++i)
    if (h[2 * i + 1] >= h[2 * i]) {
      ev.emplace_back(h[2 * i], 1 + kind[i]);
      ev.emplace_back(h[2 * i + 1], -(1 + kind[i]));
    }
  if (ev.empty()) return "";
  std::sort(ev.begin(), ev.end());
  int cnt[5] = {0, 0, 0, 0, 0};
  double busy = 0, gemm = 0, panel = 0, small = 0, leaves_only = 0, lu_only = 0;
  for (size_t i = 0; i + 1 < ev.size(); ++i) {
    const int k = std::abs(ev[i].second) - 1;
    cnt[k] += ev[i].second > 0 ? 1 : -1;
    const double dt = (double)(ev[i + 1].first - ev[i].first) * 1e-6;
    const bool any_update = cnt[kSlotGemm] + cnt[kSlotPanel] + cnt[kSlotSmall] > 0;
    if (cnt[0] + cnt[1] + cnt[2] + cnt[3] + cnt[4] > 0) busy += dt;
    if (cnt[kSlotGemm] > 0) gemm += dt;
    if (cnt[kSlotGemm] == 0 && cnt[kSlotPanel] > 0) panel += dt;
    if (cnt[kSlotGemm] == 0 && cnt[kSlotPanel] == 0 && cnt[kSlotSmall] > 0) small += dt;
    if (!any_update && cnt[kSlotLuLeaf] + cnt[kSlotSolveLeaf] > 0) leaves_only += dt;
    if (!any_update && cnt[kSlotLuLeaf] > 0) lu_only += dt;
  }
  const double span = (double)(ev.back().first - ev.front().first) * 1e-6;
  char note[384];
  std::snprintf(note, sizeof note,
                "factorisation timeline: %.1f ms from first start to last end; a BF16 tensor-core GEMM running %.1f "
                "ms, else a TF32 panel update %.1f ms, else a small FP32 update %.1f ms, only leaves %.1f ms (an LU "
                "leaf %.1f ms), nothing %.1f ms",
                span, gemm, panel, small, leaves_only, lu_only, span - busy);
  return note;
}

std::string size_class(int m, int n, int k) {
  auto c = [](int v) { return v <= 256 ? "S" : (v <= 2048 ? "M" : "L"); };
  return std::string("gemm ") + c(m) + c(n) + c(k);
}

}  // namespace

struct MixedSolver::Impl {
  CallProfile prof;
  alignas(64) unsigned char map_a[kTensorMapBytes], map_b[kTensorMapBytes];
  long op_ld = 0;      // leading dimension of both BF16 operand buffers (elements)
  int op_rows = 0;     // rows of both operand buffers
  const void* map_key[2] = {};      // the buffers the tensor maps describe
  cudaGraphExec_t graph = nullptr;  // the captured factorisation
  const void* graph_key[8] = {};
  int graph_n = 0;
  size_t graph_kernels = 0;
  // per-launch device stamps of the GEMMs (live timing that works inside the graph): slots taken in
  // launch order as the recursion runs (or is captured), with each launch's flops
  std::string host_note;  // host-side times of the last build (allocations, graph capture)
  int used_slots = 0;     // GEMM stamp slots and work of the last build
  double used_work = 0;
  Buf stamps;
  int slot_cap = 0, nslots = 0;
  double slot_work = 0;  // GEMM flops
  std::vector<unsigned char> slot_kind;  // kSlot* of each slot, in launch order
  std::vector<double> slot_flop;         // and its flops
  int graph_slots = 0;
  double graph_work = 0;
  // the solve's buffers for q right-hand sides per pass (GMRES vectors, FP32 preconditioner
  // vectors, split-solve scratch, mat-vec partials, dot partials)
  void reserve_solve(int q, cudaStream_t s) {
    const size_t blk = (size_t)n3 * q;
    const bool fresh = !trsv.p || trsv.bytes < trsv_scratch_bytes(n3);
    trsv.ensure(trsv_scratch_bytes(n3), "solve scratch");
    if (fresh) ck(cudaMemsetAsync(trsv.p, 0, trsv.bytes, s), "solve scratch clear");  // flags start at 0
    vecs.ensure(blk * (4 + (krylov + 1) + krylov) * sizeof(double), "GMRES vectors");
    zf.ensure(blk * sizeof(float), "preconditioner vectors (FP32)");
    part.ensure((size_t)32 * 16 * n3 * sizeof(double), "residual partials");
    pdots.ensure((size_t)std::min(4 * sms, (n3 + 255) / 256) * 32 * 16 * sizeof(double), "dot partials");
    dots.ensure(32 * 16 * sizeof(double), "dots");
  }
  unsigned long long* next_stamp(double flops, unsigned char kind = kSlotGemm) {
    if (nslots >= slot_cap) return nullptr;
    if (kind == kSlotGemm) slot_work += flops;
    slot_kind.push_back(kind);
    slot_flop.push_back(flops);
    return stamps.as<unsigned long long>() + 2 * (size_t)nslots++;
  }
  int n3 = 0;
  long ld32 = 0;
  double* gr64 = nullptr;  // the FP64 matrix (owned by the caller)
  long ld64 = 0;
  double tol = 1e-12;
  int max_restarts = 8, krylov = 10;
  int sms = 148;
  // second stream and fork/join events: the two triangular-solve chains of each recursion step
  // (U12 and L21) write disjoint blocks and run side by side; not with operand copies, whose
  // buffers the products of both chains would share
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool fork = false;
  Buf lu32, at, bt, status, part, pdots, dots, trsv, vecs, dl32, du32, zf;
  Buf wl32, wu32;  // the preconditioner's chain data per triangle (weights, FP16 copy of the off-diagonal blocks)
  // BF16 mirrors of the factors (L part row-major, U part column-major), written by the triangular
  // solve leaves as the entries become final; the GEMMs read their operands there by position, so no
  // operand copies are made.  Used when the GPU has room for them (4 n^2 bytes), else copies.
  Buf am, bm;
  bool mirrors = false;
  long ldm = 0;
  alignas(64) unsigned char map_am[kTensorMapBytes], map_bm[kTensorMapBytes];
  alignas(64) unsigned char map_mst[2 * kTensorMapBytes];  // the leaves' TMA stores into the mirrors
  const void* mirror_key[2] = {};
  // the triangular-solve leaves on the tensor cores (TF32): tensor maps over the factor and the
  // diagonal-block inverses; the FP32 CUDA-core leaves when BEST_GPU_SIMT_LEAVES is set
  bool tc_leaves = true;
  alignas(64) unsigned char map_leaf[kPanelMaps * kTensorMapBytes];
  const void* leaf_key[4] = {};
  // the inverses of the 256 x 256 diagonal blocks (k_combine256, one slot per 128 rows) for the
  // 256-deep leaves; has256[b]: formed for the block at row 128 b in this factorisation
  Buf dl256, du256;
  alignas(64) unsigned char map_t256[2 * kTensorMapBytes];
  const void* t256_key[2] = {};
  std::vector<char> has256;
  int* d_status() { return status.as<int>(); }
  __nv_bfloat16* am_at(int r, int c) const { return am.as<__nv_bfloat16>() + (size_t)r * ldm + c; }
  __nv_bfloat16* bm_at(int r, int c) const { return bm.as<__nv_bfloat16>() + (size_t)c * ldm + r; }

  // C = block (cr, cc) of the matrix, m x n, -= A (block (ar, ac), m x k) B (block (br, bc), k x n),
  // BF16 tensor cores: operands from the mirrors by position, or copied into the operand buffers
  void gemm(int m, int n, int k, int ar, int ac, int br, int bc, int cr, int cc, cudaStream_t s) {
    if (m <= 0 || n <= 0 || k <= 0) return;
    float* C = at_(cr, cc);
    if (tc_leaves && panel_update(m, n, k)) {
      // one side at most 128 (at most 256 with the other at most 3,840: wider, the BF16 GEMM is
      // faster than two row groups): the TF32 panel product, the narrow operand resident
      prof.begin(m <= n ? "panel update (TF32, left)" : "panel update (TF32, right)", 2.0 * m * n * k, s);
      if (m <= n)
        ck(panel_tf32(true, true, map_leaf, kMapMN, kMapK, nullptr, ar, ac, br, bc, m, n, C, ld32, cr, cc, nullptr, 0,
                      d_status(), s,
                      next_stamp(2.0 * m * n * k, kSlotPanel)),
           "panel update launch");
      else
        ck(panel_tf32(false, true, map_leaf, kMapK, kMapMN, nullptr, br, bc, ar, ac, n, m, C, ld32, cr, cc, nullptr, 0,
                      d_status(), s,
                      next_stamp(2.0 * m * n * k, kSlotPanel)),
           "panel update launch");
      prof.end(s);
      return;
    }
    if (!tc_leaves && small_update(m, n, k)) {
      prof.begin("small update (FP32 cores)", 2.0 * m * n * k, s);
      ck(launch_dependent(k_sgemm_small_minus, dim3((m + 63) / 64, (n + 63) / 64), dim3(256), 0, s, m, n, k,
                          (const float*)at_(ar, ac), (long)ld32, (const float*)at_(br, bc), (long)ld32, C, (long)ld32,
                          next_stamp(2.0 * m * n * k, kSlotSmall)),
         "small update launch");
      prof.end(s);
      BGPU_COUNT_LAUNCH();
      ck(cudaGetLastError(), "small update");
      return;
    }
    if (mirrors) {
      prof.begin(size_class(m, n, k), 2.0 * m * n * k, s);
      ck(gemm_bf16_tc_minus_at(m, n, k, map_am, ar, ac, map_bm, bc, br, C, ld32, d_status(), s,
                               next_stamp(2.0 * m * n * k), tc_leaves ? map_leaf + kMapC * kTensorMapBytes : nullptr,
                               cr, cc),
         "tensor-core GEMM");
      prof.end(s);
      return;
    }
    if (round_up(k, 64) > op_ld) throw std::runtime_error("GEMM deeper than its operand buffers");
    // operand buffers of op_rows rows: products with more rows or columns go in blocks of that size
    for (int m0 = 0; m0 < m; m0 += op_rows) {
      const int mm = std::min(op_rows, m - m0);
      prof.begin("casts", 0, s);
      ck(cast_transpose_bf16(at_(ar + m0, ac), ld32, mm, k, at.p, op_ld, s), "cast A");
      prof.end(s);
      for (int n0 = 0; n0 < n; n0 += op_rows) {
        const int nn = std::min(op_rows, n - n0);
        prof.begin("casts", 0, s);
        ck(cast_bf16(at_(br, bc + n0), ld32, k, nn, bt.p, op_ld, s), "cast B");
        prof.end(s);
        prof.begin(size_class(mm, nn, k), 2.0 * mm * nn * k, s);
        ck(gemm_bf16_tc_minus_maps(mm, nn, k, map_a, map_b, at_(cr + m0, cc + n0), ld32, d_status(), s,
                                   next_stamp(2.0 * mm * nn * k)),
           "tensor-core GEMM");
        prof.end(s);
      }
    }
  }

  static int split(int sz) {
    int h = (sz / 2) / kLeaf * kLeaf;
    return std::max(h, kLeaf);
  }

  float* at_(int r, int c) const { return lu32.as<float>() + r + (size_t)c * ld32; }

  // rows [kd, kd+h) x columns [c0, c0+w) := L^-1 (that block), L the unit lower triangle at (kd, kd)
  void trsm_llu(int kd, int h, int c0, int w, cudaStream_t s) {
    if (h <= 0 || w <= 0) return;
    if (tc_leaves && h == 256 && has256[kd / kLeaf]) {
      __nv_bfloat16* mir = mirrors ? bm_at(kd, c0) : nullptr;
      prof.begin("trsm leaf 256 (left)", 2.0 * h * h * w, s);
      ck(leaf256_tf32(true, map_leaf, map_t256, mir ? map_mst : nullptr, kd / kLeaf, kd, c0, h, w, at_(kd, c0), ld32,
                      mir, ldm, d_status(), s, next_stamp(2.0 * h * h * w, kSlotSolveLeaf)),
         "trsm leaf launch");
      prof.end(s);
      return;
    }
    if (h <= kLeaf) {
      const float* dinv = dl32.as<float>() + (size_t)(kd / kLeaf) * kLeaf * kLeaf;
      __nv_bfloat16* mir = mirrors ? bm_at(kd, c0) : nullptr;
      prof.begin(w >= kWideLeaf ? "trsm leaf (left, wide)" : "trsm leaf (left)", 2.0 * h * h * w, s);
      if (tc_leaves)
        ck(panel_tf32(true, false, map_leaf, kMapDL, kMapK, mir ? map_mst : nullptr, 0, kd, kd, c0, h, w, at_(kd, c0),
                      ld32, kd, c0, mir, ldm,
                      d_status(), s, next_stamp(2.0 * h * h * w, kSlotSolveLeaf)),
           "trsm leaf launch");
      else if (w >= kWideLeaf)
        launch_dependent(k_leaf_mult<true>, dim3((w + 127) / 128), dim3(256), (size_t)2 * 128 * kLm * sizeof(float),
                         s, dinv, h, at_(kd, c0), ld32, w, mir, ldm, next_stamp(2.0 * h * h * w, kSlotSolveLeaf));
      else
        launch_narrow_leaf<true>(dinv, h, at_(kd, c0), ld32, w, mir, ldm, sms, s,
                                 next_stamp(2.0 * h * h * w, kSlotSolveLeaf));
      prof.end(s);
      BGPU_COUNT_LAUNCH();
      ck(cudaGetLastError(), "trsm leaf");
      return;
    }
    const int h1 = split(h);
    trsm_llu(kd, h1, c0, w, s);
    gemm(h - h1, w, h1, kd + h1, kd, kd, c0, kd + h1, c0, s);
    trsm_llu(kd + h1, h - h1, c0, w, s);
  }

  // rows [r0, r0+m) x columns [kd, kd+h) := (that block) U^-1, U the upper triangle at (kd, kd)
  void trsm_ru(int kd, int h, int r0, int m, cudaStream_t s) {
    if (h <= 0 || m <= 0) return;
    if (tc_leaves && h == 256 && has256[kd / kLeaf]) {
      __nv_bfloat16* mir = mirrors ? am_at(r0, kd) : nullptr;
      prof.begin("trsm leaf 256 (right)", 2.0 * h * h * m, s);
      ck(leaf256_tf32(false, map_leaf, map_t256, mir ? map_mst : nullptr, kd / kLeaf, kd, r0, h, m, at_(r0, kd), ld32,
                      mir, ldm, d_status(), s, next_stamp(2.0 * h * h * m, kSlotSolveLeaf)),
         "trsm leaf launch");
      prof.end(s);
      return;
    }
    if (h <= kLeaf) {
      const float* dinv = du32.as<float>() + (size_t)(kd / kLeaf) * kLeaf * kLeaf;
      __nv_bfloat16* mir = mirrors ? am_at(r0, kd) : nullptr;
      prof.begin(m >= kWideLeaf ? "trsm leaf (right, wide)" : "trsm leaf (right)", 2.0 * h * h * m, s);
      if (tc_leaves)
        ck(panel_tf32(false, false, map_leaf, kMapDU, kMapMN, mir ? map_mst : nullptr, 0, kd, r0, kd, h, m, at_(r0, kd),
                      ld32, r0, kd, mir, ldm,
                      d_status(), s, next_stamp(2.0 * h * h * m, kSlotSolveLeaf)),
           "trsm leaf launch");
      else if (m >= kWideLeaf)
        launch_dependent(k_leaf_mult<false>, dim3((m + 127) / 128), dim3(256), (size_t)2 * 128 * kLm * sizeof(float),
                         s, dinv, h, at_(r0, kd), ld32, m, mir, ldm, next_stamp(2.0 * h * h * m, kSlotSolveLeaf));
      else
        launch_narrow_leaf<false>(dinv, h, at_(r0, kd), ld32, m, mir, ldm, sms, s,
                                  next_stamp(2.0 * h * h * m, kSlotSolveLeaf));
      prof.end(s);
      BGPU_COUNT_LAUNCH();
      ck(cudaGetLastError(), "trsm leaf");
      return;
    }
    const int h1 = split(h);
    trsm_ru(kd, h1, r0, m, s);
    gemm(m, h - h1, h1, r0, kd, kd, kd + h1, r0, kd + h1, s);
    trsm_ru(kd + h1, h - h1, r0, m, s);
  }

  // factors the square block at (k0, k0) of size sz in place; each 128 x 128 diagonal leaf is
  // inverted (both triangles) right after it is factored, for the triangular-solve leaves above it
  void rlu(int k0, int sz, cudaStream_t s) {
    if (sz <= kLeaf) {
      const size_t smem = (size_t)3 * 128 * kS * sizeof(float);
      const size_t off = (size_t)(k0 / kLeaf) * kLeaf * kLeaf;
      prof.begin("LU leaf + inverses", 0, s);
      launch_dependent(k_lu32_leaf_inv, dim3(1), dim3(512), smem, s, at_(k0, k0), ld32, sz, dl32.as<float>() + off,
                       du32.as<float>() + off, d_status(), next_stamp(0, kSlotLuLeaf));
      prof.end(s);
      BGPU_COUNT_LAUNCH();
      ck(cudaGetLastError(), "LU leaf");
      return;
    }
    const int h = split(sz), r = sz - h;
    rlu(k0, h, s);
    if (fork) {
      ck(cudaEventRecord(ev_fork, s), "fork");
      ck(cudaStreamWaitEvent(side, ev_fork, 0), "fork");
      trsm_llu(k0, h, k0 + h, r, s);     // U12
      trsm_ru(k0, h, k0 + h, r, side);   // L21
      ck(cudaEventRecord(ev_join, side), "join");
      ck(cudaStreamWaitEvent(s, ev_join, 0), "join");
    } else {
      trsm_llu(k0, h, k0 + h, r, s);   // U12
      trsm_ru(k0, h, k0 + h, r, s);    // L21
    }
    gemm(r, r, h, k0 + h, k0, k0, k0 + h, k0 + h, k0 + h, s);
    rlu(k0 + h, r, s);
    if (tc_leaves && sz == 256) {
      // the 256 x 256 block's inverses, for the 256-deep leaves below it
      prof.begin("256-block inverses", 0, s);
      ck(launch_dependent(k_combine256, dim3(8, 2), dim3(256), kCombineSmem, s, (const float*)lu32.as<float>(),
                          (long)ld32, k0, (const float*)dl32.as<float>(), (const float*)du32.as<float>(),
                          dl256.as<float>(), du256.as<float>(), next_stamp(0, kSlotLuLeaf)),
         "256-block inverses");
      prof.end(s);
      BGPU_COUNT_LAUNCH();
      has256[k0 / kLeaf] = 1;
    }
  }

  // Y (n3 x q, ldy) = beta Y + alpha GR X
  void matvec(const double* X, long ldx, int q, double* Y, long ldy, double alpha, double beta, cudaStream_t s) {
    // 128 threads per block, four rows each; 32 column splits at the LU's orders (fewer blocks
    // would leave SMs idle, more only add partial sums)
    const int rb = (n3 + 511) / 512;
    const int splits = std::max(1, std::min(32, (4 * sms * 8 + rb - 1) / rb));
    const int per = (n3 + splits - 1) / splits;
    part.ensure((size_t)splits * 16 * n3 * sizeof(double), "residual partials");
    if (q <= 8) {
      k_matvec64_part<8><<<dim3(rb, splits), 128, 0, s>>>(gr64, ld64, n3, X, ldx, q, per, part.as<double>());
      BGPU_COUNT_LAUNCH();
      k_matvec64_reduce<8><<<(n3 + 255) / 256, 256, 0, s>>>(part.as<double>(), n3, q, splits, alpha, beta, Y, ldy);
    } else {
      k_matvec64_part<16><<<dim3(rb, splits), 128, 0, s>>>(gr64, ld64, n3, X, ldx, q, per, part.as<double>());
      BGPU_COUNT_LAUNCH();
      k_matvec64_reduce<16><<<(n3 + 255) / 256, 256, 0, s>>>(part.as<double>(), n3, q, splits, alpha, beta, Y, ldy);
    }
    BGPU_COUNT_LAUNCH();
    ck(cudaGetLastError(), "FP64 residual");
  }

  // host copy of V_i[c] . W[c] for i < nv (nv x q values, row i)
  std::vector<double> dot(const double* V, int nv, const double* W, int q, cudaStream_t s) {
    const int blocks = std::min(4 * sms, (n3 + 255) / 256);
    pdots.ensure((size_t)blocks * 32 * 16 * sizeof(double), "dot partials");  // nv <= 17
    dots.ensure(32 * 16 * sizeof(double), "dots");
    k_dots<<<dim3(blocks, nv), 256, 0, s>>>(V, nv, W, n3, q, pdots.as<double>());
    BGPU_COUNT_LAUNCH();
    k_dots_reduce<<<(nv * q + 127) / 128, 128, 0, s>>>(pdots.as<double>(), blocks, nv * q, dots.as<double>());
    BGPU_COUNT_LAUNCH();
    std::vector<double> h((size_t)nv * q);
    ck(cudaMemcpyAsync(h.data(), dots.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "dot read");
    ck(cudaStreamSynchronize(s), "dot sync");
    return h;
  }
};

cudaError_t combine256(const float* LU, long lda, int k0, const float* DL, const float* DU, float* TL, float* TU,
                       cudaStream_t s) {
  if (k0 < 0 || k0 % 128) return cudaErrorInvalidValue;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_combine256, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCombineSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_combine256<<<dim3(8, 2), 256, kCombineSmem, s>>>(LU, lda, k0, DL, DU, TL, TU, nullptr);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t lu32_leaf(float* A, long lda, int h, float* DL, float* DU, int* status, cudaStream_t s) {
  if (h <= 0 || h > 128 || lda < h) return cudaErrorInvalidValue;
  static bool attr = false;
  const size_t smem = (size_t)3 * 128 * kS * sizeof(float);
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_lu32_leaf_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_lu32_leaf_inv<<<1, 512, smem, s>>>(A, lda, h, DL, DU, status, nullptr);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

std::vector<std::string> MixedSolver::profile_report() {
  std::vector<std::string> out = p_->prof.report();
  if (!p_->host_note.empty()) out.push_back(p_->host_note);
  p_->host_note.clear();
  return out;
}

MixedSolver::MixedSolver() : p_(new Impl) {
  const char* e = std::getenv("BEST_GPU_PROFILE");
  p_->prof.on = e && *e && std::string(e) != "0";
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&p_->sms, cudaDevAttrMultiProcessorCount, dev);
  p_->status.ensure(256, "status");
  ck(cudaMemset(p_->status.p, 0, 256), "status clear");
}
MixedSolver::~MixedSolver() {
  if (p_->graph) cudaGraphExecDestroy(p_->graph);
  if (p_->side) cudaStreamDestroy(p_->side);
  if (p_->ev_fork) cudaEventDestroy(p_->ev_fork);
  if (p_->ev_join) cudaEventDestroy(p_->ev_join);
  delete p_;
}
void MixedSolver::set_refinement(int max_restarts, int krylov) {
  p_->max_restarts = std::max(0, max_restarts);
  p_->krylov = std::min(16, std::max(1, krylov));
}
const char* MixedSolver::name() const { return "BF16 tensor-core (FP32 factors) + FP64 GMRES-IR"; }

void MixedSolver::build(const DevMesh& m, const DevDeflation& d, double* gr64, long ld, double eps, cudaStream_t s,
                        cudaEvent_t ev_assembled, cudaEvent_t ev_factored, bool wait) {
  Impl& P = *p_;
  using clk = std::chrono::steady_clock;
  const auto ms_since = [](clk::time_point t) {
    return std::chrono::duration<double, std::milli>(clk::now() - t).count();
  };
  const clk::time_point t_begin = clk::now();
  double ms_alloc = 0, ms_capture = 0, ms_inst = 0;
  P.n3 = 3 * m.n;
  // columns 128-byte aligned, but not a multiple of 1 KB apart: the triangular solves read 64
  // columns at once, and a power-of-two-like stride puts them all on the same memory partitions
  P.ld32 = round_up(P.n3, 32);
  if ((P.ld32 * 4) % 1024 == 0) P.ld32 += 32;
  P.gr64 = gr64;
  P.ld64 = ld;
  P.tol = std::max(1e-15, std::min(0.1 * eps, 1e-12));
  // (+256 bytes: the solve leaves read whole 16-byte groups at the end of the last column)
  P.lu32.ensure((size_t)P.ld32 * P.n3 * sizeof(float) + 256, "FP32 copy of GR");
  ck(cudaMemsetAsync(P.status.p, 0, sizeof(int), s), "status clear");
  ck(launch_assemble_fast(m, 0, m.n, 0, m.n, gr64, ld, d, P.lu32.as<float>(), P.ld32, s), "assembly");
  ck(cudaEventRecord(ev_assembled, s), "event");
  // everything else is allocated while the GPU assembles: the factorisation's buffers and the
  // solve's scratch (for up to 16 right-hand sides per pass)
  P.dl32.ensure(diag_inverse_elems(P.n3) * sizeof(float), "diagonal-block inverses (L)");
  P.du32.ensure(diag_inverse_elems(P.n3) * sizeof(float), "diagonal-block inverses (U)");
  // the preconditioner's chain data (weights and the FP16 copy of the off-diagonal blocks, half the
  // FP32 factor's size); without room for it the preconditioner runs without the chain
  try {
    P.wl32.ensure(chain_weights_elems(P.n3) * sizeof(float), "preconditioner chain data (L)");
    P.wu32.ensure(chain_weights_elems(P.n3) * sizeof(float), "preconditioner chain data (U)");
  } catch (const std::runtime_error&) {
    P.wl32.release();
    P.wu32.release();
  }
  P.tc_leaves = std::getenv("BEST_GPU_SIMT_LEAVES") == nullptr;
  if (P.tc_leaves && (P.leaf_key[0] != P.lu32.p || P.leaf_key[1] != P.dl32.p || P.leaf_key[2] != P.du32.p ||
                      P.leaf_key[3] != reinterpret_cast<const void*>((uintptr_t)P.n3))) {
    if (!tc_panel_maps(P.lu32.as<float>(), P.n3, P.ld32, P.dl32.as<float>(), P.du32.as<float>(), P.map_leaf))
      throw std::runtime_error("cannot build the tensor maps of the triangular-solve leaves");
    P.leaf_key[0] = P.lu32.p;
    P.leaf_key[1] = P.dl32.p;
    P.leaf_key[2] = P.du32.p;
    P.leaf_key[3] = reinterpret_cast<const void*>((uintptr_t)P.n3);
  }
  if (P.tc_leaves) {
    const int slots = (P.n3 + kLeaf - 1) / kLeaf;
    P.dl256.ensure((size_t)slots * 65536 * sizeof(float), "256-block inverses (L)");
    P.du256.ensure((size_t)slots * 65536 * sizeof(float), "256-block inverses (U)");
    if (P.t256_key[0] != P.dl256.p || P.t256_key[1] != P.du256.p) {
      if (!tc_leaf256_maps(P.dl256.as<float>(), P.du256.as<float>(), (int)(P.dl256.bytes / (65536 * sizeof(float))),
                           P.map_t256))
        throw std::runtime_error("cannot build the tensor maps of the 256-block inverses");
      P.t256_key[0] = P.dl256.p;
      P.t256_key[1] = P.du256.p;
    }
  }
  // BF16 mirrors when they fit with 4 GB to spare, else operand copies per product
  const long ldm = round_up(P.n3, 64);
  const size_t mirror_bytes = (size_t)P.n3 * ldm * 2;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t held = (P.am.p ? P.am.bytes : 0) + (P.bm.p ? P.bm.bytes : 0);
  P.mirrors = free_b + held >= 2 * mirror_bytes + ((size_t)4 << 30) && std::getenv("BEST_GPU_NO_MIRRORS") == nullptr;
  if (P.mirrors) {
    P.am.ensure(mirror_bytes, "BF16 mirror (L)");
    P.bm.ensure(mirror_bytes, "BF16 mirror (U)");
    if (P.ldm != ldm || P.mirror_key[0] != P.am.p || P.mirror_key[1] != P.bm.p) {
      if (!tc_mirror_maps(P.am.p, P.bm.p, P.n3, ldm, P.map_am, P.map_bm) ||
          !tc_mirror_store_maps(P.am.p, P.bm.p, P.n3, ldm, P.map_mst))
        throw std::runtime_error("cannot build the tensor maps of the BF16 mirrors");
      P.ldm = ldm;
      P.mirror_key[0] = P.am.p;
      P.mirror_key[1] = P.bm.p;
    }
  } else {
    // K of any product is at most about n/2; rows per buffer as many as fit beside everything else
    // (3 GB kept for the solve's scratch and vectors), at most n/2
    const long half = P.n3 / 2 + 128;
    const long op_ld = round_up(half, 64);
    const size_t held_ops = (P.at.p ? P.at.bytes : 0) + (P.bt.p ? P.bt.bytes : 0);
    const size_t avail = free_b + held_ops > ((size_t)3 << 30) ? free_b + held_ops - ((size_t)3 << 30) : 0;
    long rows = std::min<long>(half, (long)(avail / 2 / ((size_t)op_ld * 2)));
    if (const char* e = std::getenv("BEST_GPU_OPERAND_ROWS")) rows = std::min<long>(rows, std::max(256L, atol(e)));
    rows = rows >= half ? half : rows / 256 * 256;
    if (rows < 256) throw std::runtime_error("no room on the GPU for the BF16 operand buffers");
    P.at.ensure((size_t)rows * op_ld * 2, "BF16 operand A");
    P.bt.ensure((size_t)rows * op_ld * 2, "BF16 operand B");
    if (P.op_ld != op_ld || P.op_rows != (int)rows || P.map_key[0] != P.at.p || P.map_key[1] != P.bt.p) {
      if (!tc_operand_maps(P.at.p, (int)rows, op_ld, P.bt.p, (int)rows, op_ld, P.map_a, P.map_b))
        throw std::runtime_error("cannot build the tensor maps of the BF16 operands");
      P.op_ld = op_ld;
      P.op_rows = (int)rows;
      P.map_key[0] = P.at.p;
      P.map_key[1] = P.bt.p;
    }
  }
  ck(tc_gemm_prepare(), "tensor-core GEMM attributes");
  ck(cudaFuncSetAttribute(k_combine256, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCombineSmem),
     "256-block inverse attributes");
  static bool attrs = false;
  if (!attrs) {
    const int big = 200 * 1024;
    ck(cudaFuncSetAttribute(k_lu32_leaf_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024), "attr");
    ck(cudaFuncSetAttribute(k_leaf_mult<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    ck(cudaFuncSetAttribute(k_leaf_mult<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    ck(cudaFuncSetAttribute(k_apply_inv_left<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    ck(cudaFuncSetAttribute(k_apply_inv_left<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    ck(cudaFuncSetAttribute(k_apply_inv_left<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    ck(cudaFuncSetAttribute(k_apply_inv_right<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    ck(cudaFuncSetAttribute(k_apply_inv_right<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    ck(cudaFuncSetAttribute(k_apply_inv_right<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big), "attr");
    attrs = true;
  }
  P.reserve_solve(16, s);
  ms_alloc = ms_since(t_begin);
  // GEMM stamp slots: far more than the recursion's launches (about 8 per 128-row leaf with the
  // mirrors; the blocked products without them add a few per leaf)
  const int cap = 64 * ((P.n3 + kLeaf - 1) / kLeaf) + 4096;
  if (P.slot_cap < cap || !P.stamps.p) {
    P.stamps.ensure((size_t)cap * 2 * sizeof(unsigned long long), "GEMM timing stamps");
    P.slot_cap = cap;
  }
  if (!P.side) {
    ck(cudaStreamCreateWithFlags(&P.side, cudaStreamNonBlocking), "side stream");
    ck(cudaEventCreateWithFlags(&P.ev_fork, cudaEventDisableTiming), "fork event");
    ck(cudaEventCreateWithFlags(&P.ev_join, cudaEventDisableTiming), "join event");
  }
  int used_slots = 0;
  double used_work = 0;
  if (P.prof.on) {
    P.fork = false;
    P.nslots = 0;
    P.slot_work = 0;
    P.slot_kind.clear();
    P.slot_flop.clear();
    P.has256.assign((size_t)(P.n3 + kLeaf - 1) / kLeaf, 0);
    ck(stamps_reset(P.stamps.as<unsigned long long>(), P.slot_cap, s), "stamps");
    P.rlu(0, P.n3, s);  // direct launches in order, each timed
    if (P.wl32.p)
      ck(chain_weights32(P.lu32.as<float>(), P.ld32, P.dl32.as<float>(), P.du32.as<float>(), P.n3, P.wl32.as<float>(),
                         P.wu32.as<float>(), s),
         "chain weights");
    used_slots = P.nslots;
    used_work = P.slot_work;
  } else {
    // the recursion's launches depend only on the order and the buffers: capture them once as a
    // CUDA graph and replay it
    const void* key[8] = {P.lu32.p, P.mirrors ? P.am.p : P.at.p, P.mirrors ? P.bm.p : P.bt.p,
                          P.dl32.p, P.du32.p, P.stamps.p, P.wl32.p, P.tc_leaves ? P.dl256.p : nullptr};
    if (!P.graph || P.graph_n != P.n3 || !std::equal(key, key + 8, P.graph_key)) {
      const clk::time_point t_cap = clk::now();
      if (P.graph) cudaGraphExecDestroy(P.graph);
      P.graph = nullptr;
      cudaStream_t cs;
      ck(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
      cudaGraph_t g = nullptr;
      const unsigned long long launches0 = g_launches;  // captured launches do not run now
      ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
      P.fork = P.mirrors && std::getenv("BEST_GPU_ONE_STREAM") == nullptr;
      P.nslots = 0;
      P.slot_work = 0;
      P.slot_kind.clear();
      P.slot_flop.clear();
      P.has256.assign((size_t)(P.n3 + kLeaf - 1) / kLeaf, 0);
      try {
        P.rlu(0, P.n3, cs);
        if (P.wl32.p)
          ck(chain_weights32(P.lu32.as<float>(), P.ld32, P.dl32.as<float>(), P.du32.as<float>(), P.n3,
                             P.wl32.as<float>(), P.wu32.as<float>(), cs),
             "chain weights");
      } catch (...) {
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        g_launches = launches0;
        throw;
      }
      ck(cudaStreamEndCapture(cs, &g), "end capture");
      P.graph_kernels = (size_t)(g_launches - launches0);
      g_launches = launches0;
      ms_capture = ms_since(t_cap);
      const clk::time_point t_inst = clk::now();
      ck(cudaGraphInstantiate(&P.graph, g, 0), "graph instantiate");
      ms_inst = ms_since(t_inst);
      cudaGraphDestroy(g);
      cudaStreamDestroy(cs);
      std::copy(key, key + 8, P.graph_key);
      P.graph_n = P.n3;
      P.graph_slots = P.nslots;
      P.graph_work = P.slot_work;
    }
    ck(stamps_reset(P.stamps.as<unsigned long long>(), P.graph_slots, s), "stamps");
    ck(cudaGraphLaunch(P.graph, s), "graph launch");
    g_launches += P.graph_kernels;
    used_slots = P.graph_slots;
    used_work = P.graph_work;
  }
  ck(cudaEventRecord(ev_factored, s), "event");
  P.used_slots = used_slots;
  P.used_work = used_work;
  {
    char note[256];
    std::snprintf(note, sizeof note,
                  "mixed build, host side: allocations %.1f ms, graph capture %.1f ms, instantiation %.1f ms, "
                  "enqueue %.1f ms",
                  ms_alloc, ms_capture, ms_inst, ms_since(t_begin));
    P.host_note = note;
  }
  if (wait) finish_build(s);
}

size_t MixedSolver::device_bytes() const {
  const Impl& P = *p_;
  size_t b = 0;
  for (const Buf* q : {&P.stamps, &P.lu32, &P.at, &P.bt, &P.status, &P.part, &P.pdots, &P.dots, &P.trsv, &P.vecs,
                       &P.dl32, &P.du32, &P.zf, &P.wl32, &P.wu32, &P.am, &P.bm, &P.dl256, &P.du256})
    b += q->p ? q->bytes : 0;
  return b;
}

void MixedSolver::finish_build(cudaStream_t s) {
  Impl& P = *p_;
  // (the status is read after the wait: a copy to pageable host memory would block the enqueue)
  ck(cudaStreamSynchronize(s), "factorisation");
  int st = 0;
  ck(cudaMemcpyAsync(&st, P.status.p, sizeof(int), cudaMemcpyDeviceToHost, s), "status read");
  ck(cudaStreamSynchronize(s), "status read");
  const int used_slots = P.used_slots;
  const double used_work = P.used_work;
  KernelTimer& kt = kernel_timer(1);
  if (kt.on && used_slots > 0) {
    // live GEMM time of this factorisation: each launch's last end minus its first start
    std::vector<unsigned long long> h((size_t)2 * used_slots);
    ck(cudaMemcpy(h.data(), P.stamps.p, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost), "stamps");
    double ns = 0;
    int gemms = 0;
    for (int i = 0; i < used_slots; ++i)
      if (P.slot_kind[i] == kSlotGemm && h[2 * i + 1] >= h[2 * i]) {
        ns += (double)(h[2 * i + 1] - h[2 * i]);
        ++gemms;
      }
    kt.add(gemms, ns * 1e-6, used_work);
    const std::string tl = timeline_note(h, P.slot_kind, used_slots);
    if (!tl.empty()) P.host_note += "; " + tl;
    // BEST_GPU_TIMELINE=<file>: every stamped launch of this factorisation appended as
    // "slot,kind,flops,start_ns,end_ns" (kinds: 0 BF16 GEMM, 1 LU leaf, 2 triangular-solve leaf,
    // 3 small FP32 update, 4 TF32 panel update)
    if (const char* path = std::getenv("BEST_GPU_TIMELINE")) {
      if (FILE* f = std::fopen(path, "a")) {
        for (int i = 0; i < used_slots && i < (int)P.slot_kind.size(); ++i)
          std::fprintf(f, "%d,%d,%.0f,%llu,%llu\n", i, (int)P.slot_kind[i], P.slot_flop[i], h[2 * i], h[2 * i + 1]);
        std::fclose(f);
      }
    }
  }
  if (st != 0) {
    ck(cudaMemsetAsync(P.status.p, 0, sizeof(int), s), "status clear");
    throw MixedFailure(st == kZeroPivot ? "the unpivoted FP32 factorisation met a zero or non-finite pivot"
                                        : "a device-side wait ran out in the tensor-core factorisation");
  }
}

void MixedSolver::solve(int nrhs, double* d_b, long ldb, cudaStream_t s, MixedReport* rep) {
  Impl& P = *p_;
  const int n = P.n3;
  const int m = P.krylov;           // Krylov vectors per restart
  const int max_restarts = P.max_restarts;
  int total_iters = 0;
  double worst = 0.0;
  using clk = std::chrono::steady_clock;
  const clk::time_point t_begin = clk::now();
  double ms_alloc = 0;
  const bool fresh_scratch = !P.trsv.p || P.trsv.bytes < trsv_scratch_bytes(n);
  P.trsv.ensure(trsv_scratch_bytes(n), "solve scratch");
  if (fresh_scratch) ck(cudaMemsetAsync(P.trsv.p, 0, P.trsv.bytes, s), "solve scratch clear");  // flags start at 0
  for (int c0 = 0; c0 < nrhs; c0 += 16) {
    const int q = std::min(16, nrhs - c0);
    const size_t blk = (size_t)n * q;
    // [B | X | R | W | V_0..V_m | Z_0..Z_{m-1}]
    P.vecs.ensure(blk * (4 + (m + 1) + m) * sizeof(double), "GMRES vectors");
    P.zf.ensure(blk * sizeof(float), "preconditioner vectors (FP32)");
    if (c0 == 0) ms_alloc = std::chrono::duration<double, std::milli>(clk::now() - t_begin).count();
    double* B = P.vecs.as<double>();
    double* X = B + blk;
    double* R = X + blk;
    double* W = R + blk;
    double* V = W + blk;
    double* Z = V + (size_t)(m + 1) * blk;
    const int grid = std::min(4 * P.sms, (n + 255) / 256);
    k_copy_in<<<grid, 256, 0, s>>>(d_b + (size_t)c0 * ldb, ldb, n, q, B);
    BGPU_COUNT_LAUNCH();
    ck(cudaMemsetAsync(X, 0, blk * sizeof(double), s), "x clear");
    std::vector<double> bn2 = P.dot(B, 1, B, q, s);
    std::vector<double> bn(q);
    for (int c = 0; c < q; ++c) bn[c] = std::sqrt(bn2[c]);
    double rel = 1.0;
    for (int restart = 0; restart <= max_restarts; ++restart) {
      // R = B - GR X
      ck(cudaMemcpyAsync(R, B, blk * sizeof(double), cudaMemcpyDeviceToDevice, s), "r copy");
      if (restart > 0) {
        P.prof.begin("FP64 mat-vec", 2.0 * n * (double)n * q, s);
        P.matvec(X, n, q, R, n, -1.0, 1.0, s);
        P.prof.end(s);
      }
      std::vector<double> rn2 = P.dot(R, 1, R, q, s);
      std::vector<double> rn(q), inv(q);
      rel = 0.0;
      for (int c = 0; c < q; ++c) {
        rn[c] = std::sqrt(rn2[c]);
        const double r = bn[c] > 0 ? rn[c] / bn[c] : 0.0;
        rel = std::max(rel, std::isnan(r) ? INFINITY : r);
        inv[c] = rn[c] > 0 ? 1.0 / rn[c] : 0.0;
      }
      if (rel <= P.tol || restart == max_restarts) break;
      ck(cudaMemcpyAsync(P.dots.p, inv.data(), q * sizeof(double), cudaMemcpyHostToDevice, s), "scale");
      k_scale_cols<<<grid, 256, 0, s>>>(R, P.dots.as<double>(), V, n, q);
      BGPU_COUNT_LAUNCH();
      // Arnoldi with Givens rotations, per column
      std::vector<std::vector<double>> H(q, std::vector<double>((size_t)(m + 1) * m, 0.0));
      std::vector<std::vector<double>> cs(q, std::vector<double>(m)), sn(q, std::vector<double>(m));
      std::vector<std::vector<double>> g(q, std::vector<double>(m + 1, 0.0));
      for (int c = 0; c < q; ++c) g[c][0] = rn[c];
      int jdone = 0;
      std::vector<double> coef((size_t)(m + 1) * q);
      for (int j = 0; j < m; ++j) {
        double* Vj = V + (size_t)j * blk;
        double* Zj = Z + (size_t)j * blk;
        P.prof.begin("preconditioner solve", 0, s);
        k_to_f32<<<grid, 256, 0, s>>>(Vj, blk, P.zf.as<float>());
        BGPU_COUNT_LAUNCH();
        ck(trsv_lu32_inv(P.lu32.as<float>(), P.ld32, P.dl32.as<float>(), P.du32.as<float>(), P.wl32.as<float>(),
                         P.wu32.as<float>(), n, P.zf.as<float>(), n, q, P.trsv.p, P.d_status(), s),
           "preconditioner");
        k_to_f64<<<grid, 256, 0, s>>>(P.zf.as<float>(), blk, Zj);
        BGPU_COUNT_LAUNCH();
        P.prof.end(s);
        P.prof.begin("FP64 mat-vec", 2.0 * n * (double)n * q, s);
        P.matvec(Zj, n, q, W, n, 1.0, 0.0, s);
        P.prof.end(s);
        // classical Gram-Schmidt, twice
        std::vector<double> h = P.dot(V, j + 1, W, q, s);
        ck(cudaMemcpyAsync(P.dots.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s), "coef");
        k_combine<<<grid, 256, 0, s>>>(V, j + 1, P.dots.as<double>(), -1.0, W, n, q);
        BGPU_COUNT_LAUNCH();
        std::vector<double> h2 = P.dot(V, j + 1, W, q, s);
        ck(cudaMemcpyAsync(P.dots.p, h2.data(), h2.size() * sizeof(double), cudaMemcpyHostToDevice, s), "coef");
        k_combine<<<grid, 256, 0, s>>>(V, j + 1, P.dots.as<double>(), -1.0, W, n, q);
        BGPU_COUNT_LAUNCH();
        for (size_t t = 0; t < h.size(); ++t) h[t] += h2[t];
        std::vector<double> wn2 = P.dot(W, 1, W, q, s);
        std::vector<double> sc(q);
        double est = 0.0;
        for (int c = 0; c < q; ++c) {
          const double hn = std::sqrt(wn2[c]);
          sc[c] = hn > 0 ? 1.0 / hn : 0.0;
          double* Hc = H[c].data();
          for (int i = 0; i <= j; ++i) Hc[i * m + j] = h[(size_t)i * q + c];
          Hc[(j + 1) * m + j] = hn;
          for (int i = 0; i < j; ++i) {
            const double a = Hc[i * m + j], b = Hc[(i + 1) * m + j];
            Hc[i * m + j] = cs[c][i] * a + sn[c][i] * b;
            Hc[(i + 1) * m + j] = -sn[c][i] * a + cs[c][i] * b;
          }
          const double a = Hc[j * m + j], b = Hc[(j + 1) * m + j];
          const double rr = std::hypot(a, b);
          cs[c][j] = rr > 0 ? a / rr : 1.0;
          sn[c][j] = rr > 0 ? b / rr : 0.0;
          Hc[j * m + j] = rr;
          Hc[(j + 1) * m + j] = 0.0;
          g[c][j + 1] = -sn[c][j] * g[c][j];
          g[c][j] = cs[c][j] * g[c][j];
          if (bn[c] > 0) est = std::max(est, std::fabs(g[c][j + 1]) / bn[c]);
        }
        ck(cudaMemcpyAsync(P.dots.p, sc.data(), q * sizeof(double), cudaMemcpyHostToDevice, s), "scale");
        k_scale_cols<<<grid, 256, 0, s>>>(W, P.dots.as<double>(), V + (size_t)(j + 1) * blk, n, q);
        BGPU_COUNT_LAUNCH();
        ++total_iters;
        jdone = j + 1;
        if (est <= 0.5 * P.tol) break;
      }
      // y from the triangular H, then X += Z y
      for (int c = 0; c < q; ++c) {
        std::vector<double> y(jdone, 0.0);
        for (int i = jdone - 1; i >= 0; --i) {
          double v = g[c][i];
          for (int k = i + 1; k < jdone; ++k) v -= H[c][i * m + k] * y[k];
          y[i] = H[c][i * m + i] != 0 ? v / H[c][i * m + i] : 0.0;
        }
        for (int i = 0; i < jdone; ++i) coef[(size_t)i * q + c] = y[i];
      }
      ck(cudaMemcpyAsync(P.dots.p, coef.data(), (size_t)jdone * q * sizeof(double), cudaMemcpyHostToDevice, s),
         "coef");
      k_combine<<<grid, 256, 0, s>>>(Z, jdone, P.dots.as<double>(), 1.0, X, n, q);
      BGPU_COUNT_LAUNCH();
    }
    int st = 0;
    ck(cudaMemcpyAsync(&st, P.status.p, sizeof(int), cudaMemcpyDeviceToHost, s), "status read");
    ck(cudaStreamSynchronize(s), "solve");
    if (st != 0) {
      ck(cudaMemsetAsync(P.status.p, 0, sizeof(int), s), "status clear");
      throw MixedFailure("a device-side wait ran out in the refined solve");
    }
    if (!(rel <= P.tol)) throw MixedFailure("GMRES refinement did not reach the requested residual");
    k_copy_out<<<grid, 256, 0, s>>>(X, n, q, d_b + (size_t)c0 * ldb, ldb);
    BGPU_COUNT_LAUNCH();
    ck(cudaGetLastError(), "copy out");
    worst = std::max(worst, rel);
  }
  if (rep) {
    rep->iterations = total_iters;
    rep->relres = worst;
  }
  char note[160];
  std::snprintf(note, sizeof note, "mixed solve, host side: allocations %.1f ms, whole call %.1f ms", ms_alloc,
                std::chrono::duration<double, std::milli>(clk::now() - t_begin).count());
  P.host_note = note;
}

}  // namespace bgpu
