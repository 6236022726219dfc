// FP64 LU factorisation with partial pivoting for BEST's GR (dgetrf semantics), on the B200.
//
// What it replaces: LAPACK dgetrf(nar3, nar3, GR, nar3, ipiv, info), best/best.f:444, error
// handling best/best.f:458-468.
//
// Structure (right-looking, blocked, recursive panels):
//   for each block column of nb columns:
//     panel     recursive split down to leaves of <= 32 columns; a leaf is one cooperative
//               kernel (k_leaf) whose CTAs each hold a slice of the leaf's rows in shared memory
//               and agree on each pivot through a bounded grid barrier (one barrier per column)
//     laswp     the panel's row interchanges on the other columns (k_laswp)
//     trsm      U12 = L11^-1 A12, recursive: 32-row leaves (k_trsm_leaf) + GEMM updates
//     gemm      A22 -= L21 U12 on the FP64 tensor cores (mma.sync m8n8k4 f64, cp.async pipeline)
// tcgen05 has no FP64 kind, so the FP64 trailing update runs on DMMA; the mixed-precision path
// (lu_mixed.cu) puts its trailing update on tcgen05.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "bgpu_internal.h"

namespace bgpu {

unsigned long long g_launches = 0;

namespace {

// ------------------------------------------------------------------------------------------
// small PTX helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// ------------------------------------------------------------------------------------------
// DGEMM: C(m x n) -= A(m x k) B(k x n), column-major, on DMMA
// ------------------------------------------------------------------------------------------
// CTA tile BM x BN, K step BK, warp tile WM x WN made of 8x8 DMMA fragments.  Shared memory:
//   As[stage][BK][BM + 4]  (A's columns are contiguous in m; +4 doubles makes the fragment loads of
//                           a half-warp hit 16 distinct 8-byte banks)
//   Bs[stage][BN][BK + 4]  (B's columns are contiguous in k)
template <int BM, int BN, int BK, int WM, int WN, int STAGES>
struct GemmCfg {
  static constexpr int kWarpsM = BM / WM, kWarpsN = BN / WN;
  static constexpr int kThreads = kWarpsM * kWarpsN * 32;
  static constexpr int kFm = WM / 8, kFn = WN / 8;
  static constexpr int kAStride = BM + 4, kBStride = BK + 4;
  static constexpr int kAStage = BK * kAStride, kBStage = BN * kBStride;
  static constexpr size_t kSmem = (size_t)STAGES * (kAStage + kBStage) * sizeof(double);
};

template <int BM, int BN, int BK, int WM, int WN, int STAGES>
__global__ void __launch_bounds__(GemmCfg<BM, BN, BK, WM, WN, STAGES>::kThreads)
    k_dgemm_nn_minus(int m, int n, int k, const double* __restrict__ A, long lda, const double* __restrict__ B,
                     long ldb, double* __restrict__ C, long ldc) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, STAGES>;
  extern __shared__ __align__(16) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * Cfg::kAStage;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp % Cfg::kWarpsM) * WM, wn0 = (warp / Cfg::kWarpsM) * WN;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int ktiles = (k + BK - 1) / BK;

  auto load_stage = [&](int stage, int kt) {
    const int k0 = kt * BK;
    double* as = As + stage * Cfg::kAStage;
    double* bs = Bs + stage * Cfg::kBStage;
    // A: BK columns of BM rows, 2 doubles per 16-byte copy
    for (int c = tid; c < BK * (BM / 2); c += Cfg::kThreads) {
      const int kk = c / (BM / 2), mm = (c % (BM / 2)) * 2;
      const int gr = m0 + mm, gk = k0 + kk;
      int bytes = 0;
      if (gk < k) bytes = (gr + 1 < m) ? 16 : (gr < m ? 8 : 0);
      const double* src = bytes ? A + (size_t)gk * lda + gr : A;
      cp_async16(as + kk * Cfg::kAStride + mm, src, bytes);
    }
    // B: BN columns of BK rows
    for (int c = tid; c < BN * (BK / 2); c += Cfg::kThreads) {
      const int nn = c / (BK / 2), kk = (c % (BK / 2)) * 2;
      const int gc = n0 + nn, gk = k0 + kk;
      int bytes = 0;
      if (gc < n) bytes = (gk + 1 < k) ? 16 : (gk < k ? 8 : 0);
      const double* src = bytes ? B + (size_t)gc * ldb + gk : B;
      cp_async16(bs + nn * Cfg::kBStride + kk, src, bytes);
    }
  };

  double acc[Cfg::kFm][Cfg::kFn][2];
#pragma unroll
  for (int i = 0; i < Cfg::kFm; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::kFn; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < ktiles) load_stage(nk % STAGES, nk);
      cp_async_commit();
    }
    const double* as = As + (kt % STAGES) * Cfg::kAStage;
    const double* bs = Bs + (kt % STAGES) * Cfg::kBStage;
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double af[Cfg::kFm], bf[Cfg::kFn];
#pragma unroll
      for (int i = 0; i < Cfg::kFm; ++i) af[i] = as[(k4 + (lane & 3)) * Cfg::kAStride + wm0 + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < Cfg::kFn; ++j) bf[j] = bs[(wn0 + j * 8 + (lane >> 2)) * Cfg::kBStride + k4 + (lane & 3)];
#pragma unroll
      for (int i = 0; i < Cfg::kFm; ++i)
#pragma unroll
        for (int j = 0; j < Cfg::kFn; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();
  // epilogue: C -= acc; fragment element (row lane/4, cols 2*(lane%4) + {0,1})
#pragma unroll
  for (int i = 0; i < Cfg::kFm; ++i) {
    const int gr = m0 + wm0 + i * 8 + (lane >> 2);
    if (gr >= m) continue;
#pragma unroll
    for (int j = 0; j < Cfg::kFn; ++j) {
      const int gc = n0 + wn0 + j * 8 + 2 * (lane & 3);
      if (gc < n) {
        double* p = C + (size_t)gc * ldc + gr;
        *p = *p - acc[i][j][0];
      }
      if (gc + 1 < n) {
        double* p = C + (size_t)(gc + 1) * ldc + gr;
        *p = *p - acc[i][j][1];
      }
    }
  }
}

using GemmBig = GemmCfg<128, 128, 16, 32, 64, 4>;
using GemmSmall = GemmCfg<64, 64, 16, 32, 32, 4>;

template <int BM, int BN, int BK, int WM, int WN, int ST>
cudaError_t run_gemm(int m, int n, int k, const double* A, long lda, const double* B, long ldb, double* C, long ldc,
                     cudaStream_t s) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, ST>;
  static bool attr_set = false;
  auto kern = k_dgemm_nn_minus<BM, BN, BK, WM, WN, ST>;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  dim3 grid((m + BM - 1) / BM, (n + BN - 1) / BN);
  kern<<<grid, Cfg::kThreads, Cfg::kSmem, s>>>(m, n, k, A, lda, B, ldb, C, ldc);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// Leaf panel factorisation: m x w (w <= 32), partial pivoting, cooperative over G CTAs
// ------------------------------------------------------------------------------------------
constexpr int kLeafW = 32;
constexpr int kLeafThreads = 256;
constexpr unsigned kSpinLimit = 1u << 22;  // polls of a barrier word before giving up (~0.3 s)

struct LeafScratchLayout {
  // offsets in bytes from the scratch base
  static constexpr size_t kBarrier = 0;                    // unsigned counter
  static constexpr size_t kCand = 256;                     // [2][kMaxCta] {double val; long long idx}
  static constexpr int kMaxCta = 256;
  static constexpr size_t kCandRows = kCand + 2 * kMaxCta * 16;           // [2][kMaxCta][kLeafW] double
  static constexpr size_t kRowJ = kCandRows + 2 * kMaxCta * kLeafW * 8;   // [2][kLeafW] double
  static constexpr size_t kEnd = kRowJ + 2 * kLeafW * 8;
};

// Waits until every CTA of the grid has arrived here `round` times.  Returns false, with the status
// word set, when the wait runs out (the caller then returns; every other CTA's wait runs out too).
__device__ bool grid_barrier(unsigned* counter, unsigned expected, int* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    atomicAdd(counter, 1u);
    unsigned spins = 0;
    while (ld_acquire_u32(counter) < expected) {
      if (++spins > kSpinLimit) {
        atomicExch(status, (int)kWaitTimeout);
        ok = 0;
        break;
      }
      __nanosleep(40);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

struct Cand {
  double val;
  long long idx;
};

// rows of the leaf held by each CTA: R (the last CTA may hold fewer); shared: sp[c * R + r]
__global__ void __launch_bounds__(kLeafThreads) k_leaf(double* __restrict__ P, long lda, int m, int w, int R,
                                                       int* __restrict__ ipiv, int rowoff, int* info, int* status,
                                                       unsigned char* scratch) {
  extern __shared__ __align__(16) double sp[];
  __shared__ double s_prow[kLeafW];
  __shared__ double s_rowj[kLeafW];
  __shared__ double s_rv[kLeafThreads / 32];
  __shared__ long long s_ri[kLeafThreads / 32];
  __shared__ long long s_piv;
  __shared__ int s_win;
  __shared__ double s_pval;

  const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + LeafScratchLayout::kBarrier);
  Cand* cand = reinterpret_cast<Cand*>(scratch + LeafScratchLayout::kCand);
  double* cand_rows = reinterpret_cast<double*>(scratch + LeafScratchLayout::kCandRows);
  double* rowj = reinterpret_cast<double*>(scratch + LeafScratchLayout::kRowJ);
  constexpr int kMax = LeafScratchLayout::kMaxCta;

  const int rbeg = cta * R;
  const int nr = max(0, min(m, rbeg + R) - rbeg);
  for (int idx = tid; idx < nr * w; idx += kLeafThreads) {
    const int r = idx % nr, c = idx / nr;
    sp[c * R + r] = P[(size_t)c * lda + rbeg + r];
  }
  __syncthreads();

  unsigned rounds = 0;
  for (int j = 0; j < w && j < m; ++j) {
    const int par = j & 1;
    // local candidate: max |P(i, j)| over rows i >= j, first index on ties
    double bv = -1.0;
    long long bi = 0x7fffffffffffffffLL;
    for (int r = tid; r < nr; r += kLeafThreads) {
      const int i = rbeg + r;
      if (i < j) continue;
      const double v = fabs(sp[j * R + r]);
      if (v > bv || (v == bv && i < bi)) {
        bv = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) {
        bv = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      s_rv[warp] = bv;
      s_ri[warp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      for (int q = 1; q < kLeafThreads / 32; ++q)
        if (s_rv[q] > bv || (s_rv[q] == bv && s_ri[q] < bi)) {
          bv = s_rv[q];
          bi = s_ri[q];
        }
      s_rv[0] = bv;
      s_ri[0] = bi;
    }
    __syncthreads();
    bv = s_rv[0];
    bi = s_ri[0];

    if (G > 1) {
      // publish the candidate, its row, and (owner of row j) row j; then one barrier
      if (tid == 0) {
        cand[par * kMax + cta].val = bv;
        cand[par * kMax + cta].idx = bi;
      }
      if (tid < w && bi != 0x7fffffffffffffffLL) cand_rows[((size_t)par * kMax + cta) * kLeafW + tid] = sp[tid * R + (int)(bi - rbeg)];
      if (j >= rbeg && j < rbeg + nr && tid < w) rowj[par * kLeafW + tid] = sp[tid * R + (j - rbeg)];
      ++rounds;
      if (!grid_barrier(counter, rounds * (unsigned)G, status)) return;
      // global pivot
      if (warp == 0) {
        double gv = -1.0;
        long long gi = 0x7fffffffffffffffLL;
        int gw = 0;
        for (int q = lane; q < G; q += 32) {
          const double v = __ldcg(&cand[par * kMax + q].val);
          const long long i = __ldcg(&cand[par * kMax + q].idx);
          if (v > gv || (v == gv && i < gi)) {
            gv = v;
            gi = i;
            gw = q;
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, gv, o);
          const long long oi = __shfl_xor_sync(0xffffffffu, gi, o);
          const int ow = __shfl_xor_sync(0xffffffffu, gw, o);
          if (ov > gv || (ov == gv && oi < gi)) {
            gv = ov;
            gi = oi;
            gw = ow;
          }
        }
        if (lane == 0) {
          s_piv = gi;
          s_win = gw;
        }
      }
      __syncthreads();
      if (tid < w) {
        s_prow[tid] = __ldcg(&cand_rows[((size_t)par * kMax + s_win) * kLeafW + tid]);
        s_rowj[tid] = __ldcg(&rowj[par * kLeafW + tid]);
      }
    } else {
      if (tid == 0) s_piv = bi;
      __syncthreads();
      if (tid < w) {
        s_prow[tid] = sp[tid * R + (int)(s_piv - rbeg)];
        s_rowj[tid] = sp[tid * R + j];
      }
    }
    __syncthreads();
    const int p = (int)s_piv;
    if (tid == 0) s_pval = s_prow[j];
    if (cta == 0 && tid == 0) {
      ipiv[j] = rowoff + p + 1;
      if (s_prow[j] == 0.0) atomicCAS(info, 0, rowoff + j + 1);
    }
    __syncthreads();
    const double pv = s_pval;
    if (pv != 0.0) {
      // interchange rows j and p inside the panel
      if (p != j) {
        if (j >= rbeg && j < rbeg + nr && tid < w) sp[tid * R + (j - rbeg)] = s_prow[tid];
        if (p >= rbeg && p < rbeg + nr && tid < w) sp[tid * R + (p - rbeg)] = s_rowj[tid];
      }
      __syncthreads();
      // scale the column below the pivot and update the rest of the leaf
      const double rp = 1.0 / pv;
      for (int r = tid; r < nr; r += kLeafThreads) {
        const int i = rbeg + r;
        if (i <= j) continue;
        const double l = sp[j * R + r] * rp;
        sp[j * R + r] = l;
        for (int c = j + 1; c < w; ++c) sp[c * R + r] -= l * s_prow[c];
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < nr * w; idx += kLeafThreads) {
    const int r = idx % nr, c = idx / nr;
    P[(size_t)c * lda + rbeg + r] = sp[c * R + r];
  }
}

// ------------------------------------------------------------------------------------------
// Row interchanges on columns [c0, c1): for j in [j0, j1) swap rows j and ipiv[j]-1 (in order)
// ------------------------------------------------------------------------------------------
__global__ void k_laswp(double* __restrict__ A, long lda, int c0, int c1, const int* __restrict__ ipiv, int j0,
                        int j1) {
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = c < c1;
  double* col = A + (size_t)(act ? c : c0) * lda;
  for (int j = j0; j < j1; ++j) {
    const int p = ipiv[j] - 1;  // uniform across the block: no divergence
    if (p != j && act) {
      const double t = col[j];
      col[j] = col[p];
      col[p] = t;
    }
  }
}

// ------------------------------------------------------------------------------------------
// TRSM leaf: B(kb x nc) := L^-1 B, L unit lower kb x kb (kb <= 32); one CTA per 64 columns
// ------------------------------------------------------------------------------------------
constexpr int kTrsmLeaf = 32;
constexpr int kTrsmCols = 64;
__global__ void __launch_bounds__(kTrsmCols) k_trsm_leaf(const double* __restrict__ L, long ldl, int kb,
                                                          double* __restrict__ B, long ldb, int nc) {
  __shared__ double sl[kTrsmLeaf][kTrsmLeaf + 1];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kb * kb; idx += kTrsmCols) {
    const int r = idx % kb, c = idx / kb;
    sl[r][c] = L[(size_t)c * ldl + r];
  }
  __syncthreads();
  const int col = blockIdx.x * kTrsmCols + tid;
  if (col >= nc) return;
  double x[kTrsmLeaf];
  double* b = B + (size_t)col * ldb;
#pragma unroll
  for (int r = 0; r < kTrsmLeaf; ++r)
    if (r < kb) x[r] = b[r];
#pragma unroll
  for (int r = 0; r < kTrsmLeaf; ++r) {
    if (r < kb) {
      double v = x[r];
#pragma unroll
      for (int c = 0; c < kTrsmLeaf; ++c)
        if (c < r) v -= sl[r][c] * x[c];
      x[r] = v;
    }
  }
#pragma unroll
  for (int r = 0; r < kTrsmLeaf; ++r)
    if (r < kb) b[r] = x[r];
}

struct Ctx {
  double* A;
  long lda;
  int n;
  int* ipiv;
  int* info;
  int* status;
  unsigned char* leaf_scratch;
  int num_sms;
  cudaStream_t s;
};

cudaError_t gemm_minus(int m, int n, int k, const double* A, long lda, const double* B, long ldb, double* C, long ldc,
                       cudaStream_t s) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  const long tiles_big = (long)((m + 127) / 128) * ((n + 127) / 128);
  if (tiles_big >= 148) return run_gemm<128, 128, 16, 32, 64, 4>(m, n, k, A, lda, B, ldb, C, ldc, s);
  return run_gemm<64, 64, 16, 32, 32, 4>(m, n, k, A, lda, B, ldb, C, ldc, s);
}

cudaError_t laswp(const Ctx& c, int c0, int c1, int j0, int j1) {
  if (c1 <= c0 || j1 <= j0) return cudaSuccess;
  const int threads = 128;
  k_laswp<<<(c1 - c0 + threads - 1) / threads, threads, 0, c.s>>>(c.A, c.lda, c0, c1, c.ipiv, j0, j1);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// B(kb x nc) := L^-1 B with L unit lower (both inside A, leading dimension lda)
cudaError_t trsm_lower_unit(const double* L, long lda, int kb, double* B, int nc, cudaStream_t s) {
  if (kb <= 0 || nc <= 0) return cudaSuccess;
  if (kb <= kTrsmLeaf) {
    k_trsm_leaf<<<(nc + kTrsmCols - 1) / kTrsmCols, kTrsmCols, 0, s>>>(L, lda, kb, B, lda, nc);
    BGPU_COUNT_LAUNCH();
    return cudaGetLastError();
  }
  int k1 = (kb / 2 + 15) / 16 * 16;
  if (k1 >= kb) k1 = kb / 2;
  cudaError_t e = trsm_lower_unit(L, lda, k1, B, nc, s);
  if (e != cudaSuccess) return e;
  e = gemm_minus(kb - k1, nc, k1, L + k1, lda, B, lda, B + k1, lda, s);
  if (e != cudaSuccess) return e;
  return trsm_lower_unit(L + k1 + (size_t)k1 * lda, lda, kb - k1, B + k1, nc, s);
}

cudaError_t leaf(const Ctx& c, int k, int w) {
  const int m = c.n - k;
  int G = std::max(1, std::min(c.num_sms, (m + 255) / 256));
  G = std::min(G, LeafScratchLayout::kMaxCta);
  int R = (m + G - 1) / G;
  size_t smem = (size_t)R * w * sizeof(double);
  while (smem > 200 * 1024 && G < std::min(c.num_sms, LeafScratchLayout::kMaxCta)) {
    ++G;
    R = (m + G - 1) / G;
    smem = (size_t)R * w * sizeof(double);
  }
  if (smem > 220 * 1024) return cudaErrorInvalidValue;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_leaf, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  double* P = c.A + k + (size_t)k * c.lda;
  int* ip = c.ipiv + k;
  if (G > 1) {
    cudaError_t e = cudaMemsetAsync(c.leaf_scratch + LeafScratchLayout::kBarrier, 0, 4, c.s);
    if (e != cudaSuccess) return e;
    long lda = c.lda;
    int mm = m, ww = w, RR = R, ro = k;
    int* info = c.info;
    int* status = c.status;
    unsigned char* scr = c.leaf_scratch;
    void* args[] = {&P, &lda, &mm, &ww, &RR, &ip, &ro, &info, &status, &scr};
    BGPU_COUNT_LAUNCH();
    return cudaLaunchCooperativeKernel((const void*)k_leaf, dim3(G), dim3(kLeafThreads), args, smem, c.s);
  }
  k_leaf<<<1, kLeafThreads, smem, c.s>>>(P, c.lda, m, w, R, ip, k, c.info, c.status, c.leaf_scratch);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// columns [k, k + w), rows [k, n)
cudaError_t panel(const Ctx& c, int k, int w) {
  if (w <= kLeafW) return leaf(c, k, w);
  int w1 = (w / 2) / 8 * 8;
  if (w1 < 8) w1 = w / 2;
  cudaError_t e = panel(c, k, w1);
  if (e != cudaSuccess) return e;
  if ((e = laswp(c, k + w1, k + w, k, k + w1)) != cudaSuccess) return e;
  double* A = c.A;
  const long lda = c.lda;
  if ((e = trsm_lower_unit(A + k + (size_t)k * lda, lda, w1, A + k + (size_t)(k + w1) * lda, w - w1, c.s)) !=
      cudaSuccess)
    return e;
  if ((e = gemm_minus(c.n - k - w1, w - w1, w1, A + (k + w1) + (size_t)k * lda, lda, A + k + (size_t)(k + w1) * lda,
                      lda, A + (k + w1) + (size_t)(k + w1) * lda, lda, c.s)) != cudaSuccess)
    return e;
  if ((e = panel(c, k + w1, w - w1)) != cudaSuccess) return e;
  return laswp(c, k, k + w1, k + w1, k + w);
}

}  // namespace

// Live timing of kernel launches (opt-in; for the roofline report).

void KernelTimer::begin(cudaStream_t s) {
  if (!on) return;
  if (used == ev.size()) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    ev.emplace_back(a, b);
  }
  cudaEventRecord(ev[used].first, s);
}

void KernelTimer::end(cudaStream_t s, double w) {
  if (!on) return;
  cudaEventRecord(ev[used].second, s);
  ++used;
  work += w;
}

void KernelTimer::enable(bool v) {
  on = v;
  used = 0;
  work = 0;
}

void KernelTimer::read(int* launches, double* ms, double* w) {
  double t = 0;
  if (used) cudaEventSynchronize(ev[used - 1].second);
  for (size_t i = 0; i < used; ++i) {
    float x = 0;
    cudaEventElapsedTime(&x, ev[i].first, ev[i].second);
    t += x;
  }
  *launches = (int)used;
  *ms = t;
  *w = work;
  used = 0;
  work = 0;
}

KernelTimer& kernel_timer(int id) {
  static KernelTimer timers[kTimedKernels];
  return timers[id < 0 || id >= kTimedKernels ? 0 : id];
}

size_t lu_scratch_bytes(int) { return LeafScratchLayout::kEnd; }

cudaError_t dgemm_nn_minus(int m, int n, int k, const double* A, long lda, const double* B, long ldb, double* C,
                           long ldc, cudaStream_t s) {
  return gemm_minus(m, n, k, A, lda, B, ldb, C, ldc, s);
}

cudaError_t lu64_getrf(double* A, long lda, int n, int* ipiv, int* d_info, int* d_status, const LuScratch& ws,
                       cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (ws.bytes < LeafScratchLayout::kEnd) return cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  Ctx c{A, lda, n, ipiv, d_info, d_status, static_cast<unsigned char*>(ws.base), sms, s};
  cudaError_t e = cudaMemsetAsync(d_info, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  const int nb = 256;
  for (int k = 0; k < n; k += nb) {
    const int kb = std::min(nb, n - k);
    if ((e = panel(c, k, kb)) != cudaSuccess) return e;
    if ((e = laswp(c, k + kb, n, k, k + kb)) != cudaSuccess) return e;
    if ((e = laswp(c, 0, k, k, k + kb)) != cudaSuccess) return e;
    if (k + kb < n) {
      if ((e = trsm_lower_unit(A + k + (size_t)k * lda, lda, kb, A + k + (size_t)(k + kb) * lda, n - k - kb, s)) !=
          cudaSuccess)
        return e;
      kernel_timer(0).begin(s);
      if ((e = gemm_minus(n - k - kb, n - k - kb, kb, A + (k + kb) + (size_t)k * lda, lda,
                          A + k + (size_t)(k + kb) * lda, lda, A + (k + kb) + (size_t)(k + kb) * lda, lda, s)) !=
          cudaSuccess)
        return e;
      kernel_timer(0).end(s, 2.0 * (double)(n - k - kb) * (double)(n - k - kb) * kb);
    }
  }
  return cudaSuccess;
}

}  // namespace bgpu
