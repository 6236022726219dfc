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
// (mixed.cu, with tc_gemm.cu) puts its updates on tcgen05.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "bgpu_internal.h"

namespace bgpu {

unsigned long long g_launches = 0;

namespace {

// The LU works on a batch of independent matrices at once (one matrix is a batch of one): every
// kernel below takes per-matrix pointers and extents and finds its matrix from its block index.
constexpr int kMaxBatch = 16;

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

// A batch of independent products C_i -= A_i B_i with a common k (the same step of several LUs):
// blockIdx.z selects the product; CTAs outside a product's tiles return at once.
struct GemmItem {
  const double* A;
  const double* B;
  double* C;
  long lda, ldb, ldc;
  int m, n;
};
struct GemmBatch {
  int k;
  int count;
  GemmItem it[kMaxBatch];
};

template <int BM, int BN, int BK, int WM, int WN, int STAGES>
__global__ void __launch_bounds__(GemmCfg<BM, BN, BK, WM, WN, STAGES>::kThreads)
    k_dgemm_nn_minus(const __grid_constant__ GemmBatch gb) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, STAGES>;
  extern __shared__ __align__(16) double smem[];
  const GemmItem& g = gb.it[blockIdx.z];
  const int m = g.m, n = g.n, k = gb.k;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (m0 >= m || n0 >= n) return;
  const double* __restrict__ A = g.A;
  const double* __restrict__ B = g.B;
  double* __restrict__ C = g.C;
  const long lda = g.lda, ldb = g.ldb, ldc = g.ldc;
  double* As = smem;
  double* Bs = smem + STAGES * Cfg::kAStage;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp % Cfg::kWarpsM) * WM, wn0 = (warp / Cfg::kWarpsM) * WN;
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
    // fragments double-buffered in registers: the next k4 step's loads are issued before this
    // step's DMMAs (the accumulation order over k is the same for every tile shape)
    double af[2][Cfg::kFm], bf[2][Cfg::kFn];
#pragma unroll
    for (int i = 0; i < Cfg::kFm; ++i) af[0][i] = as[(lane & 3) * Cfg::kAStride + wm0 + i * 8 + (lane >> 2)];
#pragma unroll
    for (int j = 0; j < Cfg::kFn; ++j) bf[0][j] = bs[(wn0 + j * 8 + (lane >> 2)) * Cfg::kBStride + (lane & 3)];
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      const int cur = (k4 / 4) & 1, nxt = cur ^ 1;
      if (k4 + 4 < BK) {
#pragma unroll
        for (int i = 0; i < Cfg::kFm; ++i)
          af[nxt][i] = as[(k4 + 4 + (lane & 3)) * Cfg::kAStride + wm0 + i * 8 + (lane >> 2)];
#pragma unroll
        for (int j = 0; j < Cfg::kFn; ++j)
          bf[nxt][j] = bs[(wn0 + j * 8 + (lane >> 2)) * Cfg::kBStride + k4 + 4 + (lane & 3)];
      }
#pragma unroll
      for (int i = 0; i < Cfg::kFm; ++i)
#pragma unroll
        for (int j = 0; j < Cfg::kFn; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[cur][i], bf[cur][j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  // epilogue through shared memory (the pipeline's buffers, free now): the tile column-major
  // (stride BM + 2; fragment element (row lane/4, cols 2*(lane%4) + {0,1})), then C -= tile with
  // each column read and written by consecutive threads in 16-byte pieces
  double* ct = smem;
  constexpr int kCs = BM + 2;
  static_assert((size_t)BN * kCs <= (size_t)STAGES * (Cfg::kAStage + Cfg::kBStage), "C tile must fit");
#pragma unroll
  for (int i = 0; i < Cfg::kFm; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::kFn; ++j) {
      const int r = wm0 + i * 8 + (lane >> 2), c = wn0 + j * 8 + 2 * (lane & 3);
      ct[c * kCs + r] = acc[i][j][0];
      ct[(c + 1) * kCs + r] = acc[i][j][1];
    }
  __syncthreads();
  const bool full = m0 + BM <= m && n0 + BN <= n && (ldc % 2) == 0 && ((uintptr_t)C & 15) == 0;
  for (int e = tid; e < BN * (BM / 2); e += Cfg::kThreads) {
    const int c = e / (BM / 2), r = (e % (BM / 2)) * 2;
    const int gr = m0 + r, gc = n0 + c;
    if (full) {
      double2* p = reinterpret_cast<double2*>(C + (size_t)gc * ldc + gr);
      double2 v = *p;
      v.x = v.x - ct[c * kCs + r];
      v.y = v.y - ct[c * kCs + r + 1];
      *p = v;
    } else if (gc < n) {
      if (gr < m) C[(size_t)gc * ldc + gr] = C[(size_t)gc * ldc + gr] - ct[c * kCs + r];
      if (gr + 1 < m) C[(size_t)gc * ldc + gr + 1] = C[(size_t)gc * ldc + gr + 1] - ct[c * kCs + r + 1];
    }
  }
}

// the kernel's shared-memory attribute, once (before any stream capture)
template <int BM, int BN, int BK, int WM, int WN, int ST>
cudaError_t gemm_attr() {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, ST>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_dgemm_nn_minus<BM, BN, BK, WM, WN, ST>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  return cudaSuccess;
}

template <int BM, int BN, int BK, int WM, int WN, int ST>
cudaError_t run_gemm(const GemmBatch& gb, cudaStream_t s) {
  using Cfg = GemmCfg<BM, BN, BK, WM, WN, ST>;
  auto kern = k_dgemm_nn_minus<BM, BN, BK, WM, WN, ST>;
  cudaError_t e0 = gemm_attr<BM, BN, BK, WM, WN, ST>();
  if (e0 != cudaSuccess) return e0;
  int mm = 0, nn = 0;
  for (int i = 0; i < gb.count; ++i) {
    mm = std::max(mm, gb.it[i].m);
    nn = std::max(nn, gb.it[i].n);
  }
  dim3 grid((mm + BM - 1) / BM, (nn + BN - 1) / BN, gb.count);
  kern<<<grid, Cfg::kThreads, Cfg::kSmem, s>>>(gb);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// The DGEMM tile shapes the autotuner chooses from (all K steps of 16, 4 cp.async stages).
enum GemmShape { kShapeBig = 0, kShapeSmall, kShapeTall, kShapeWide, kNumShapes };
const char* const kShapeNames[kNumShapes] = {"128x128", "64x64", "128x64", "64x128"};

cudaError_t run_shape(int shape, const GemmBatch& gb, cudaStream_t s) {
  switch (shape) {
    case kShapeBig: return run_gemm<128, 128, 16, 32, 64, 4>(gb, s);
    case kShapeSmall: return run_gemm<64, 64, 16, 32, 32, 4>(gb, s);
    case kShapeTall: return run_gemm<128, 64, 32, 32, 32, 2>(gb, s);
    default: return run_gemm<64, 128, 16, 32, 64, 4>(gb, s);
  }
}

// ------------------------------------------------------------------------------------------
// Autotuner of the DGEMM tile shape.  Key: (ceil log2 of the largest m, of the largest n, k, batch
// count).  While tuning is on, the first product with a new key (outside stream capture) is split
// into kNumShapes slices of its columns (or rows, when it is narrow), each computed with one shape
// and timed with CUDA events; the fastest shape is kept for the key.  The product is still
// computed exactly once, and the result does not depend on the shape (every shape accumulates each
// entry over k in the same order), so tuning changes times only.  Untuned keys use the fixed rule
// (128 x 64 when that gives at least one tile per SM, else 64 x 64; the tuner's choices on B200).
// ------------------------------------------------------------------------------------------
struct Tuner {
  bool on = false;
  std::map<unsigned long long, int> choice;
  std::map<unsigned long long, std::vector<float>> times;
  cudaEvent_t ev[kNumShapes + 1] = {};
};
Tuner& tuner() {
  static Tuner t;
  return t;
}
int ceil_log2(int v) {
  int r = 0;
  while ((1 << r) < v) ++r;
  return r;
}
unsigned long long tune_key(int mm, int nn, int k, int count) {
  return ((unsigned long long)ceil_log2(mm) << 40) | ((unsigned long long)ceil_log2(nn) << 32) |
         ((unsigned long long)k << 8) | (unsigned long long)count;
}

bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &st);
  return st != cudaStreamCaptureStatusNone;
}

cudaError_t gemm_batch(const GemmBatch& gb0, cudaStream_t s) {
  GemmBatch gb;
  gb.k = gb0.k;
  gb.count = 0;
  int mm = 0, nn = 0;
  for (int i = 0; i < gb0.count; ++i)
    if (gb0.it[i].m > 0 && gb0.it[i].n > 0) {
      gb.it[gb.count++] = gb0.it[i];
      mm = std::max(mm, gb0.it[i].m);
      nn = std::max(nn, gb0.it[i].n);
    }
  if (gb.count == 0 || gb.k <= 0) return cudaSuccess;
  Tuner& T = tuner();
  const unsigned long long key = tune_key(mm, nn, gb.k, gb.count);
  auto found = T.choice.find(key);
  if (found != T.choice.end()) return run_shape(found->second, gb, s);
  const bool by_cols = nn >= kNumShapes * 128, by_rows = !by_cols && mm >= kNumShapes * 128;
  if (T.on && (by_cols || by_rows) && !capturing(s)) {
    for (int q = 0; q <= kNumShapes; ++q)
      if (!T.ev[q]) cudaEventCreate(&T.ev[q]);
    cudaError_t e = cudaEventRecord(T.ev[0], s);
    for (int sh = 0; sh < kNumShapes && e == cudaSuccess; ++sh) {
      GemmBatch part = gb;
      for (int i = 0; i < gb.count; ++i) {
        GemmItem& it = part.it[i];
        const int ext = by_cols ? it.n : it.m;
        const int chunk = (ext + kNumShapes - 1) / kNumShapes;
        const int lo = std::min(ext, sh * chunk), hi = std::min(ext, lo + chunk);
        if (by_cols) {
          it.B += (size_t)lo * it.ldb;
          it.C += (size_t)lo * it.ldc;
          it.n = hi - lo;
        } else {
          it.A += lo;
          it.C += lo;
          it.m = hi - lo;
        }
      }
      bool any = false;
      for (int i = 0; i < part.count; ++i) any = any || (part.it[i].m > 0 && part.it[i].n > 0);
      if (any) e = run_shape(sh, part, s);
      if (e == cudaSuccess) e = cudaEventRecord(T.ev[sh + 1], s);
    }
    if (e != cudaSuccess) return e;
    if ((e = cudaEventSynchronize(T.ev[kNumShapes])) != cudaSuccess) return e;
    std::vector<float> ms(kNumShapes);
    int best = 0;
    for (int sh = 0; sh < kNumShapes; ++sh) {
      cudaEventElapsedTime(&ms[sh], T.ev[sh], T.ev[sh + 1]);
      if (ms[sh] < ms[best]) best = sh;
    }
    T.choice[key] = best;
    T.times[key] = ms;
    return cudaSuccess;
  }
  const long tiles_tall = (long)((mm + 127) / 128) * ((nn + 63) / 64) * gb.count;
  return run_shape(tiles_tall >= 148 ? kShapeTall : kShapeSmall, gb, s);
}

cudaError_t gemm_minus(int m, int n, int k, const double* A, long lda, const double* B, long ldb, double* C, long ldc,
                       cudaStream_t s) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  GemmBatch gb;
  gb.k = k;
  gb.count = 1;
  gb.it[0] = GemmItem{A, B, C, lda, ldb, ldc, m, n};
  return gemm_batch(gb, s);
}

// ------------------------------------------------------------------------------------------
// Leaf panel factorisation: for each matrix of the batch, an m x w panel (w <= 32) with partial
// pivoting, cooperative over G CTAs per matrix (one grid for the whole batch)
// ------------------------------------------------------------------------------------------
constexpr int kLeafW = 32;
constexpr int kLeafThreads = 256;
constexpr unsigned kSpinLimit = 1u << 22;  // polls of a barrier word before giving up (~0.3 s)

struct LeafScratchLayout {
  // offsets in bytes from the scratch base
  static constexpr size_t kBarrier = 0;                    // unsigned counter
  static constexpr size_t kCand = 256;                     // [2][kMaxCta] {double val; long long idx}
  static constexpr int kMaxCta = 512;
  static constexpr size_t kCandRows = kCand + 2 * kMaxCta * 16;                         // [2][kMaxCta][kLeafW]
  static constexpr size_t kRowJ = kCandRows + 2 * (size_t)kMaxCta * kLeafW * 8;         // [2][kMaxBatch][kLeafW]
  static constexpr size_t kEnd = kRowJ + 2 * (size_t)kMaxBatch * kLeafW * 8;
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

struct LeafItem {
  double* P;   // the panel's (0, 0): A(k, k)
  long lda;
  int m;       // rows of the panel
  int* ipiv;   // ipiv + k
  int* info;
  int cta0;    // first CTA of this matrix and the number of its CTAs
  int G;
};
struct LeafBatch {
  int count;
  int w;       // panel width (common)
  int R;       // rows per CTA (common)
  int rowoff;  // k (common)
  LeafItem it[kMaxBatch];
};

// CTA c of matrix i holds rows [c R, c R + R) of its panel in shared memory: sp[col * R + r]
__global__ void __launch_bounds__(kLeafThreads) k_leaf(const __grid_constant__ LeafBatch lb, int* status,
                                                       unsigned char* scratch) {
  extern __shared__ __align__(16) double sp[];
  __shared__ double s_prow[kLeafW];
  __shared__ double s_rowj[kLeafW];
  __shared__ double s_rv[kLeafThreads / 32];
  __shared__ long long s_ri[kLeafThreads / 32];
  __shared__ long long s_piv;
  __shared__ int s_win;
  __shared__ double s_pval;

  const int gcta = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int item = 0;
  for (int i = 0; i < lb.count; ++i)
    if (gcta >= lb.it[i].cta0 && gcta < lb.it[i].cta0 + lb.it[i].G) item = i;
  const LeafItem& L = lb.it[item];
  double* __restrict__ P = L.P;
  const long lda = L.lda;
  const int m = L.m, w = lb.w, R = lb.R, G = L.G, cta0 = L.cta0, cta = gcta - cta0;
  const int total = gridDim.x;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + LeafScratchLayout::kBarrier);
  Cand* cand = reinterpret_cast<Cand*>(scratch + LeafScratchLayout::kCand);
  double* cand_rows = reinterpret_cast<double*>(scratch + LeafScratchLayout::kCandRows);
  double* rowj = reinterpret_cast<double*>(scratch + LeafScratchLayout::kRowJ) + (size_t)item * kLeafW;
  constexpr int kMax = LeafScratchLayout::kMaxCta;
  constexpr size_t kRowjPar = (size_t)kMaxBatch * kLeafW;

  const int rbeg = cta * R;
  const int nr = max(0, min(m, rbeg + R) - rbeg);
  for (int idx = tid; idx < nr * w; idx += kLeafThreads) {
    const int r = idx % nr, c = idx / nr;
    sp[c * R + r] = P[(size_t)c * lda + rbeg + r];
  }
  __syncthreads();

  unsigned rounds = 0;
  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    const bool live = j < m;  // (uniform for a matrix; every CTA still takes every barrier)
    // local candidate: max |P(i, j)| over rows i >= j, first index on ties
    double bv = -1.0;
    long long bi = 0x7fffffffffffffffLL;
    if (live)
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

    if (total > 1) {
      // publish the candidate, its row, and (owner of row j) row j; then one barrier
      if (tid == 0) {
        cand[par * kMax + gcta].val = bv;
        cand[par * kMax + gcta].idx = bi;
      }
      if (tid < w && bi != 0x7fffffffffffffffLL)
        cand_rows[((size_t)par * kMax + gcta) * kLeafW + tid] = sp[tid * R + (int)(bi - rbeg)];
      if (live && j >= rbeg && j < rbeg + nr && tid < w) rowj[par * kRowjPar + tid] = sp[tid * R + (j - rbeg)];
      ++rounds;
      if (!grid_barrier(counter, rounds * (unsigned)total, status)) return;
      if (!live) continue;
      // this matrix's pivot: the best of its G candidates
      if (warp == 0) {
        double gv = -1.0;
        long long gi = 0x7fffffffffffffffLL;
        int gw = 0;
        for (int q = lane; q < G; q += 32) {
          const double v = __ldcg(&cand[par * kMax + cta0 + q].val);
          const long long i = __ldcg(&cand[par * kMax + cta0 + q].idx);
          if (v > gv || (v == gv && i < gi)) {
            gv = v;
            gi = i;
            gw = cta0 + q;
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
        s_rowj[tid] = __ldcg(&rowj[par * kRowjPar + tid]);
      }
    } else {
      if (!live) break;
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
      L.ipiv[j] = lb.rowoff + p + 1;
      if (s_prow[j] == 0.0) atomicCAS(L.info, 0, lb.rowoff + j + 1);
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
// Row interchanges on columns [c0, c1_i) of each matrix: for j in [j0, j1) swap rows j and
// ipiv[j]-1 (in order); blockIdx.y selects the matrix
// ------------------------------------------------------------------------------------------
struct SwapItem {
  double* A;
  long lda;
  const int* ipiv;
  int c1;
};
struct SwapBatch {
  int count;
  SwapItem it[kMaxBatch];
};
__global__ void k_laswp(const __grid_constant__ SwapBatch sb, int c0, int j0, int j1) {
  const SwapItem& S = sb.it[blockIdx.y];
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c0 + (int)(blockIdx.x * blockDim.x) >= S.c1) return;
  const bool act = c < S.c1;
  double* col = S.A + (size_t)(act ? c : c0) * S.lda;
  for (int j = j0; j < j1; ++j) {
    const int p = S.ipiv[j] - 1;  // uniform across the block: no divergence
    if (p != j && act) {
      const double t = col[j];
      col[j] = col[p];
      col[p] = t;
    }
  }
}

// ------------------------------------------------------------------------------------------
// TRSM leaf: B(kb x nc) := L^-1 B, L unit lower kb x kb (kb <= 32), per matrix (blockIdx.y);
// one CTA per 64 columns
// ------------------------------------------------------------------------------------------
constexpr int kTrsmLeaf = 32;
constexpr int kTrsmCols = 64;
struct TriItem {
  const double* L;  // the unit lower triangle's (0, 0)
  double* B;        // the right-hand block's (0, 0)
  long ld;          // leading dimension of both
  int nc;           // columns of B
};
struct TriBatch {
  int count;
  TriItem it[kMaxBatch];
};
__global__ void __launch_bounds__(kTrsmCols) k_trsm_leaf(const __grid_constant__ TriBatch tb, int kb) {
  __shared__ double sl[kTrsmLeaf][kTrsmLeaf + 1];
  const TriItem& T = tb.it[blockIdx.y];
  if ((int)(blockIdx.x * kTrsmCols) >= T.nc) return;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kb * kb; idx += kTrsmCols) {
    const int r = idx % kb, c = idx / kb;
    sl[r][c] = T.L[(size_t)c * T.ld + r];
  }
  __syncthreads();
  const int col = blockIdx.x * kTrsmCols + tid;
  if (col >= T.nc) return;
  double x[kTrsmLeaf];
  double* b = T.B + (size_t)col * T.ld;
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

// ------------------------------------------------------------------------------------------
// Host side: the blocked recursive LU over a batch of matrices
// ------------------------------------------------------------------------------------------
struct Ctx {
  LuItem items[kMaxBatch];
  int count;
  int* status;
  unsigned char* leaf_scratch;
  int num_sms;
  cudaStream_t s;
};
// the matrices worked on together (indices into Ctx::items)
struct Group {
  int n = 0;
  int idx[kMaxBatch];
};

// B_i(kb x nc_i) := L_i^-1 B_i for every item (L unit lower, both inside the matrix)
cudaError_t trsm_lower_unit(const TriBatch& tb, int kb, cudaStream_t s) {
  if (kb <= 0 || tb.count == 0) return cudaSuccess;
  int ncmax = 0;
  for (int i = 0; i < tb.count; ++i) ncmax = std::max(ncmax, tb.it[i].nc);
  if (ncmax <= 0) return cudaSuccess;
  if (kb <= kTrsmLeaf) {
    k_trsm_leaf<<<dim3((ncmax + kTrsmCols - 1) / kTrsmCols, tb.count), kTrsmCols, 0, s>>>(tb, kb);
    BGPU_COUNT_LAUNCH();
    return cudaGetLastError();
  }
  int k1 = (kb / 2 + 15) / 16 * 16;
  if (k1 >= kb) k1 = kb / 2;
  cudaError_t e = trsm_lower_unit(tb, k1, s);
  if (e != cudaSuccess) return e;
  GemmBatch gb;
  gb.k = k1;
  gb.count = tb.count;
  TriBatch t2 = tb;
  for (int i = 0; i < tb.count; ++i) {
    const TriItem& t = tb.it[i];
    gb.it[i] = GemmItem{t.L + k1, t.B, t.B + k1, t.ld, t.ld, t.ld, kb - k1, t.nc};
    t2.it[i].L = t.L + k1 + (size_t)k1 * t.ld;
    t2.it[i].B = t.B + k1;
  }
  if ((e = gemm_batch(gb, s)) != cudaSuccess) return e;
  return trsm_lower_unit(t2, kb - k1, s);
}

// row interchanges j0..j1 on columns [c0, c1_i) with c1_i = to_n ? n_i : c1
cudaError_t laswp(const Ctx& c, const Group& g, int c0, int c1, bool to_n, int j0, int j1) {
  if (j1 <= j0) return cudaSuccess;
  SwapBatch sb;
  sb.count = 0;
  int span = 0;
  for (int q = 0; q < g.n; ++q) {
    const LuItem& it = c.items[g.idx[q]];
    const int e1 = to_n ? it.n : c1;
    if (e1 <= c0) continue;
    sb.it[sb.count++] = SwapItem{it.A, it.lda, it.ipiv, e1};
    span = std::max(span, e1 - c0);
  }
  if (sb.count == 0) return cudaSuccess;
  const int threads = 128;
  k_laswp<<<dim3((span + threads - 1) / threads, sb.count), threads, 0, c.s>>>(sb, c0, j0, j1);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// the leaves (columns [k, k + w), rows [k, n_i)) of every item of g, in as few cooperative launches
// as the co-residency of their CTAs allows
cudaError_t leaf_attr() {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_leaf, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  return cudaSuccess;
}

cudaError_t leaf(const Ctx& c, const Group& g, int k, int w) {
  if (g.n == 0) return cudaSuccess;
  cudaError_t e0 = leaf_attr();
  if (e0 != cudaSuccess) return e0;
  long total_rows = 0;
  for (int q = 0; q < g.n; ++q) total_rows += c.items[g.idx[q]].n - k;
  // rows per CTA: at least 256, enough that the CTAs fit on the GPU at once
  int R = (int)std::max<long>(256, (total_rows + c.num_sms - 1) / c.num_sms);
  for (;;) {
    const size_t smem = (size_t)R * w * sizeof(double);
    if (smem > 220 * 1024) break;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_leaf, kLeafThreads, smem) != cudaSuccess) per_sm = 1;
    long ctas = 0;
    for (int q = 0; q < g.n; ++q) ctas += (c.items[g.idx[q]].n - k + R - 1) / R;
    if (ctas <= (long)per_sm * c.num_sms && ctas <= LeafScratchLayout::kMaxCta) {
      LeafBatch lb;
      lb.count = g.n;
      lb.w = w;
      lb.R = R;
      lb.rowoff = k;
      int cta = 0;
      for (int q = 0; q < g.n; ++q) {
        const LuItem& it = c.items[g.idx[q]];
        const int m = it.n - k;
        const int G = (m + R - 1) / R;
        lb.it[q] = LeafItem{it.A + k + (size_t)k * it.lda, it.lda, m, it.ipiv + k, it.info, cta, G};
        cta += G;
      }
      int* status = c.status;
      unsigned char* scr = c.leaf_scratch;
      if (cta > 1) {
        cudaError_t e = cudaMemsetAsync(c.leaf_scratch + LeafScratchLayout::kBarrier, 0, 4, c.s);
        if (e != cudaSuccess) return e;
        void* args[] = {&lb, &status, &scr};
        BGPU_COUNT_LAUNCH();
        return cudaLaunchCooperativeKernel((const void*)k_leaf, dim3(cta), dim3(kLeafThreads), args, smem, c.s);
      }
      k_leaf<<<1, kLeafThreads, smem, c.s>>>(lb, status, scr);
      BGPU_COUNT_LAUNCH();
      return cudaGetLastError();
    }
    R += 32;
  }
  // too many rows for one co-resident grid: halves of the group, one after the other
  if (g.n == 1) return cudaErrorInvalidValue;
  Group a, b;
  for (int q = 0; q < g.n; ++q) {
    Group& t = (q < g.n / 2) ? a : b;
    t.idx[t.n++] = g.idx[q];
  }
  cudaError_t e = leaf(c, a, k, w);
  if (e != cudaSuccess) return e;
  return leaf(c, b, k, w);
}

// columns [k, k + w), rows [k, n_i) of every item of g
cudaError_t panel(const Ctx& c, const Group& g, int k, int w) {
  if (w <= kLeafW) return leaf(c, g, k, w);
  int w1 = (w / 2) / 8 * 8;
  if (w1 < 8) w1 = w / 2;
  cudaError_t e = panel(c, g, k, w1);
  if (e != cudaSuccess) return e;
  if ((e = laswp(c, g, k + w1, k + w, false, k, k + w1)) != cudaSuccess) return e;
  TriBatch tb;
  tb.count = g.n;
  GemmBatch gb;
  gb.k = w1;
  gb.count = g.n;
  for (int q = 0; q < g.n; ++q) {
    const LuItem& it = c.items[g.idx[q]];
    double* A = it.A;
    const long lda = it.lda;
    tb.it[q] = TriItem{A + k + (size_t)k * lda, A + k + (size_t)(k + w1) * lda, lda, w - w1};
    gb.it[q] = GemmItem{A + (k + w1) + (size_t)k * lda, A + k + (size_t)(k + w1) * lda,
                        A + (k + w1) + (size_t)(k + w1) * lda, lda, lda, lda, it.n - k - w1, w - w1};
  }
  if ((e = trsm_lower_unit(tb, w1, c.s)) != cudaSuccess) return e;
  if ((e = gemm_batch(gb, c.s)) != cudaSuccess) return e;
  if ((e = panel(c, g, k + w1, w - w1)) != cudaSuccess) return e;
  return laswp(c, g, k, k + w1, false, k + w1, k + w);
}

// one block column of width kb at k for the items of g (n_i - k >= kb for all of them)
cudaError_t block_step(const Ctx& c, const Group& g, int k, int kb) {
  cudaError_t e;
  if ((e = panel(c, g, k, kb)) != cudaSuccess) return e;
  if ((e = laswp(c, g, k + kb, 0, true, k, k + kb)) != cudaSuccess) return e;
  if ((e = laswp(c, g, 0, k, false, k, k + kb)) != cudaSuccess) return e;
  TriBatch tb;
  tb.count = 0;
  GemmBatch gb;
  gb.k = kb;
  gb.count = 0;
  double flops = 0;
  for (int q = 0; q < g.n; ++q) {
    const LuItem& it = c.items[g.idx[q]];
    const int rest = it.n - k - kb;
    if (rest <= 0) continue;
    double* A = it.A;
    const long lda = it.lda;
    tb.it[tb.count++] = TriItem{A + k + (size_t)k * lda, A + k + (size_t)(k + kb) * lda, lda, rest};
    gb.it[gb.count++] = GemmItem{A + (k + kb) + (size_t)k * lda, A + k + (size_t)(k + kb) * lda,
                                 A + (k + kb) + (size_t)(k + kb) * lda, lda, lda, lda, rest, rest};
    flops += 2.0 * rest * (double)rest * kb;
  }
  if (tb.count == 0) return cudaSuccess;
  if ((e = trsm_lower_unit(tb, kb, c.s)) != cudaSuccess) return e;
  kernel_timer(0).begin(c.s);
  if ((e = gemm_batch(gb, c.s)) != cudaSuccess) return e;
  kernel_timer(0).end(c.s, flops);
  return cudaSuccess;
}

constexpr int kBlock = 256;  // block-column width nb

cudaError_t getrf_batch(Ctx& c) {
  cudaError_t e;
  for (int i = 0; i < c.count; ++i)
    if ((e = cudaMemsetAsync(c.items[i].info, 0, sizeof(int), c.s)) != cudaSuccess) return e;
  int nmax = 0;
  for (int i = 0; i < c.count; ++i) nmax = std::max(nmax, c.items[i].n);
  for (int k = 0; k < nmax; k += kBlock) {
    // the items with a whole block column at k go together; an item's last, narrower block column
    // is factored on its own (so every item sees the same blocking as when factored alone)
    Group full;
    for (int i = 0; i < c.count; ++i)
      if (c.items[i].n - k >= kBlock) full.idx[full.n++] = i;
    if (full.n && (e = block_step(c, full, k, kBlock)) != cudaSuccess) return e;
    for (int i = 0; i < c.count; ++i) {
      const int kb = c.items[i].n - k;
      if (kb <= 0 || kb >= kBlock) continue;
      Group one;
      one.idx[one.n++] = i;
      if ((e = block_step(c, one, k, kb)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

int device_sms() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
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
  extra_launches = 0;
  extra_ms = 0;
}

void KernelTimer::read(int* launches, double* ms, double* w) {
  double t = 0;
  if (used) cudaEventSynchronize(ev[used - 1].second);
  for (size_t i = 0; i < used; ++i) {
    float x = 0;
    cudaEventElapsedTime(&x, ev[i].first, ev[i].second);
    t += x;
  }
  *launches = (int)used + extra_launches;
  *ms = t + extra_ms;
  *w = work;
  used = 0;
  work = 0;
  extra_launches = 0;
  extra_ms = 0;
}

KernelTimer& kernel_timer(int id) {
  static KernelTimer timers[kTimedKernels];
  return timers[id < 0 || id >= kTimedKernels ? 0 : id];
}

size_t lu_scratch_bytes(int) { return LeafScratchLayout::kEnd; }

cudaError_t dgemm_nn_minus(int m, int n, int k, const double* A, long lda, const double* B, long ldb, double* C,
                           long ldc, cudaStream_t s) {
  kernel_timer(0).begin(s);
  const cudaError_t e = gemm_minus(m, n, k, A, lda, B, ldb, C, ldc, s);
  kernel_timer(0).end(s, 2.0 * m * n * (double)k);
  return e;
}

cudaError_t lu64_getrf(double* A, long lda, int n, int* ipiv, int* d_info, int* d_status, const LuScratch& ws,
                       cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  LuItem it{A, lda, n, ipiv, d_info};
  return lu64_getrf_batch(&it, 1, d_status, ws, s);
}

cudaError_t lu64_getrf_batch(const LuItem* items, int count, int* d_status, const LuScratch& ws, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (count > kMaxBatch || ws.bytes < LeafScratchLayout::kEnd) return cudaErrorInvalidValue;
  Ctx c;
  c.count = 0;
  for (int i = 0; i < count; ++i)
    if (items[i].n > 0) c.items[c.count++] = items[i];
  c.status = d_status;
  c.leaf_scratch = static_cast<unsigned char*>(ws.base);
  c.num_sms = device_sms();
  c.s = s;
  return getrf_batch(c);
}

void lu_autotune(bool on) { tuner().on = on; }

cudaError_t lu_prepare() {
  cudaError_t e;
  if ((e = gemm_attr<128, 128, 16, 32, 64, 4>()) != cudaSuccess) return e;
  if ((e = gemm_attr<64, 64, 16, 32, 32, 4>()) != cudaSuccess) return e;
  if ((e = gemm_attr<128, 64, 32, 32, 32, 2>()) != cudaSuccess) return e;
  if ((e = gemm_attr<64, 128, 16, 32, 64, 4>()) != cudaSuccess) return e;
  return leaf_attr();
}

std::string lu_autotune_table() {
  std::string out;
  for (auto& kv : tuner().choice) {
    char buf[256];
    const unsigned long long key = kv.first;
    std::snprintf(buf, sizeof buf, "m<=2^%llu n<=2^%llu k=%llu batch=%llu: %s", (key >> 40) & 0xff, (key >> 32) & 0xff,
                  (key >> 8) & 0xffffff, key & 0xff, kShapeNames[kv.second]);
    out += buf;
    auto t = tuner().times.find(key);
    if (t != tuner().times.end()) {
      out += " (ms";
      for (float v : t->second) {
        std::snprintf(buf, sizeof buf, " %.3f", v);
        out += buf;
      }
      out += ")";
    }
    out += "\n";
  }
  return out;
}

}  // namespace bgpu
