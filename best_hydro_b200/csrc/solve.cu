// Solves with the LU factors for BEST's 6 (or 11) right-hand sides (dgetrs('N') semantics).
//
// What it replaces: dgetrs('N', n, nrhs, GR, n, ipiv, b, n, info), best/besolve.f90:132-133, and
// the H-matrix solver's bhm_solve behind the same seam (hmatrix/best_hmatrix.h:64-66).
//
// The solve reads the n x n factor once (HBM-bound).  Each triangle is one persistent kernel:
// CTAs take 64-row blocks in order from a ticket counter, stream their row of 64x64 blocks of the
// factor against the already-solved blocks of the unknowns, and publish each finished block through
// a readiness flag (release/acquire, with a bounded wait).  A block taken from the ticket counter
// only ever waits on blocks taken before it by CTAs that are already running, so the scheme cannot
// deadlock however many CTAs are resident.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <vector>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/best_gpu.h"
#include "bgpu_internal.h"

// Device scratch of bgpu_dgetrs_noalloc, for callers that cannot allocate GPU memory: 16 MiB held by
// every GPU that loads the library, until the process exits.  Host code must not use this name as
// an address (it is a host-side stand-in); the entry point below looks the device address up with
// cudaGetSymbolAddress once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[16u << 20];

namespace bgpu {
namespace {

constexpr int kBs = 64;           // rows per block
constexpr int kMaxRhs = 16;       // right-hand sides per call (kernels for 8 and 16)
constexpr int kThreads = 256;     // 4 quarter-rows of the inner dimension x 64 rows
// Polls a triangular-solve wait makes before it gives up (status kWaitTimeout, the kernel returns):
// 4,194,304 by default; bgpu_set_wait_limit changes it (0: a wait not satisfied at once gives up,
// which the tests of the failure path use).
constexpr unsigned kSpinLimitDefault = 1u << 22;
__constant__ unsigned c_spin_limit = kSpinLimitDefault;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

__global__ void k_perm_init(int* perm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = i;
}

// Composes the interchanges of ipiv (1-based, LAPACK order) into perm, chunk by chunk in shared
// memory: a chunk of C interchanges touches its own C rows and at most C rows below it.
constexpr int kPermChunk = 512;
__global__ void __launch_bounds__(1024) k_perm_compose(const int* __restrict__ ipiv, int n, int* __restrict__ perm) {
  __shared__ int s_ins[kPermChunk];   // perm values of the chunk's own rows
  __shared__ int s_tgt[kPermChunk];   // target row of each interchange
  __shared__ int s_slot[kPermChunk];  // outside target: slot of its first occurrence, else -1
  __shared__ int s_out[kPermChunk];   // perm values of outside targets (by slot)
  const int tid = threadIdx.x;
  for (int j0 = 0; j0 < n; j0 += kPermChunk) {
    const int C = min(kPermChunk, n - j0);
    const int j1 = j0 + C;
    if (tid < C) {
      s_ins[tid] = perm[j0 + tid];
      s_tgt[tid] = ipiv[j0 + tid] - 1;
    }
    __syncthreads();
    if (tid < C) {
      const int p = s_tgt[tid];
      int slot = -1;
      if (p >= j1) {
        slot = tid;
        for (int q = 0; q < tid; ++q)
          if (s_tgt[q] == p) {
            slot = q;
            break;
          }
        if (slot == tid) s_out[tid] = perm[p];
      }
      s_slot[tid] = slot;
    }
    __syncthreads();
    if (tid == 0) {
      for (int t = 0; t < C; ++t) {
        const int p = s_tgt[t];
        if (p == j0 + t) continue;
        int* a = &s_ins[t];
        int* b = (p < j1) ? &s_ins[p - j0] : &s_out[s_slot[t]];
        const int v = *a;
        *a = *b;
        *b = v;
      }
    }
    __syncthreads();
    if (tid < C) {
      perm[j0 + tid] = s_ins[tid];
      if (s_slot[tid] == tid) perm[s_tgt[tid]] = s_out[tid];
    }
    __syncthreads();
  }
}

// Y(i, r) = X(perm[i], r)
template <typename T>
__global__ void k_gather_rows(const T* __restrict__ X, long ldx, const int* __restrict__ perm, int n, int nrhs,
                              T* __restrict__ Y, long ldy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  for (int r = 0; r < nrhs; ++r) Y[(size_t)r * ldy + i] = X[(size_t)r * ldx + p];
}

template <typename T>
__global__ void k_copy_cols(const T* __restrict__ Y, long ldy, int n, int nrhs, T* __restrict__ X, long ldx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int r = 0; r < nrhs; ++r) X[(size_t)r * ldx + i] = Y[(size_t)r * ldy + i];
}

// asynchronous copy of one element global -> shared (4 or 8 bytes)
template <int B>
__device__ __forceinline__ void cp_async_elem(void* sdst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gsrc), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// the commit of a group of asynchronous copies
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// asynchronous 16-byte (both addresses 16-byte aligned) or 4-byte copies global -> shared, the
// bytes from `bytes` (0..16, or 0..4) on zero-filled, no bytes read when it is 0; `policy` an L2
// cache policy (l2_evict_first)
__device__ __forceinline__ void cp_async16z(void* sdst, const void* gsrc, int bytes, unsigned long long policy) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2, %3;\n" ::"r"(d), "l"(gsrc), "r"(bytes),
               "l"(policy)
               : "memory");
}
__device__ __forceinline__ void cp_async4z(void* sdst, const void* gsrc, int bytes, unsigned long long policy) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2, %3;\n" ::"r"(d), "l"(gsrc), "r"(bytes),
               "l"(policy)
               : "memory");
}
// an L2 policy that evicts the lines it touches first (streams read once)
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
// all but the N most recent groups of asynchronous copies complete
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Warp 0 waits until flags[jb] == epoch, then counts how many more flags in the direction `step`
// (+1 or -1) are ready too, up to 32 and within [lo, hi).  Returns that count (>= 1), or 0 when the
// wait runs out (status set).  Every thread of the block must call it.
__device__ int wait_ready(const unsigned* flags, int jb, int step, int lo, int hi, unsigned epoch, int* status,
                          int* s_cnt) {
  if (threadIdx.x < 32) {
    int cnt = 0;
    unsigned spins = 0;
    for (;;) {
      const int q = jb + step * (int)threadIdx.x;
      const bool in = q >= lo && q < hi;
      const bool rdy = in && ld_acquire_u32(flags + q) == epoch;
      const unsigned ball = __ballot_sync(0xffffffffu, rdy);
      if (ball & 1u) {
        cnt = __ffs(~ball) - 1;
        if (cnt < 0 || ball == 0xffffffffu) cnt = 32;
        break;
      }
      if (++spins > c_spin_limit) {
        if (threadIdx.x == 0) atomicExch(status, (int)kWaitTimeout);
        break;
      }
      __nanosleep(32);
    }
    if (threadIdx.x == 0) *s_cnt = cnt;
  }
  __syncthreads();
  return *s_cnt;
}

// Thread 0 waits until f[lo .. hi) all equal epoch, each wait bounded (status set, the rest skipped,
// when one runs out).  Every thread of the block must call it; false when a wait ran out.
__device__ bool wait_all(const unsigned* f, int lo, int hi, unsigned epoch, int* status, int* s_ok) {
  if (threadIdx.x == 0) {
    int ok = 1;
    for (int k = lo; k < hi && ok; ++k) {
      unsigned spins = 0;
      while (ld_acquire_u32(f + k) != epoch) {
        if (++spins > c_spin_limit) {
          atomicExch(status, (int)kWaitTimeout);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// One triangle of the solve on Y (n x nrhs <= RHS, ldy).  LOWER: unit lower L, blocks in increasing
// order; otherwise upper U (non-unit diagonal), blocks in decreasing order.  F is the factor's type.
template <typename F, bool LOWER, int RHS>
__global__ void __launch_bounds__(kThreads) k_trsv(const F* __restrict__ LU, long lda, int n, double* Y, long ldy,
                                                   int nrhs, unsigned* flags, unsigned* ticket, unsigned epoch,
                                                   int* status) {
  __shared__ double s_y[kBs][RHS];  // a solved block being consumed, later the block being solved
  // the partial sums of the four quarters, then (reusing the space) the diagonal block
  constexpr int kAccWords = 4 * kBs * RHS, kDiagWords = kBs * (kBs + 1);
  __shared__ double s_buf[kAccWords > kDiagWords ? kAccWords : kDiagWords];
  __shared__ int s_blk, s_cnt;
  double(*s_acc)[kBs][RHS] = reinterpret_cast<double(*)[kBs][RHS]>(s_buf);
  double(*s_d)[kBs + 1] = reinterpret_cast<double(*)[kBs + 1]>(s_buf);
  const int nblk = (n + kBs - 1) / kBs;
  const int tid = threadIdx.x, row = tid & (kBs - 1), quarter = tid >> 6;

  for (;;) {
    if (tid == 0) s_blk = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int t = s_blk;
    if (t >= nblk) return;
    const int blk = LOWER ? t : nblk - 1 - t;
    const int r0 = blk * kBs, nr = min(kBs, n - r0);
    double acc[RHS];
#pragma unroll
    for (int r = 0; r < RHS; ++r) acc[r] = 0.0;

    // off-diagonal blocks: jb = 0 .. blk-1 (lower) or jb = nblk-1 .. blk+1 (upper)
    const int nq = LOWER ? blk : nblk - 1 - blk;
    int confirmed = 0;  // blocks known ready, counted along the processing order
    for (int q = 0; q < nq; ++q) {
      const int jb = LOWER ? q : nblk - 1 - q;
      if (q >= confirmed) {
        const int c = LOWER ? wait_ready(flags, jb, +1, 0, blk, epoch, status, &s_cnt)
                            : wait_ready(flags, jb, -1, blk + 1, nblk, epoch, status, &s_cnt);
        if (c == 0) return;
        confirmed = q + c;
      }
      const int c0 = jb * kBs, nc = min(kBs, n - c0);
      for (int idx = tid; idx < kBs * RHS; idx += kThreads) {
        const int rr = idx / RHS, r = idx % RHS;
        s_y[rr][r] = (rr < nc && r < nrhs) ? __ldcg(&Y[(size_t)r * ldy + c0 + rr]) : 0.0;
      }
      __syncthreads();
      if (row < nr) {
        const F* col = LU + (size_t)(c0 + quarter * 16) * lda + r0 + row;
#pragma unroll 4
        for (int kk = 0; kk < 16; ++kk) {
          const int cc = quarter * 16 + kk;
          if (cc < nc) {
            const double l = (double)col[(size_t)kk * lda];
#pragma unroll
            for (int r = 0; r < RHS; ++r) acc[r] -= l * s_y[cc][r];
          }
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < RHS; ++r) s_acc[quarter][row][r] = acc[r];
    __syncthreads();
    // s_y := b - sum of the off-diagonal products
    for (int idx = tid; idx < kBs * RHS; idx += kThreads) {
      const int rr = idx / RHS, r = idx % RHS;
      double v = 0.0;
      if (rr < nr && r < nrhs)
        v = Y[(size_t)r * ldy + r0 + rr] + ((s_acc[0][rr][r] + s_acc[1][rr][r]) + (s_acc[2][rr][r] + s_acc[3][rr][r]));
      s_y[rr][r] = v;
    }
    __syncthreads();
    for (int idx = tid; idx < kBs * kBs; idx += kThreads) {
      const int rr = idx % kBs, cc = idx / kBs;
      s_d[rr][cc] = (rr < nr && cc < nr) ? (double)LU[(size_t)(r0 + cc) * lda + r0 + rr] : 0.0;
    }
    __syncthreads();
    // substitution inside the diagonal block, column by column
    if (LOWER) {
      for (int c = 0; c < nr; ++c) {
        for (int idx = tid; idx < kBs * RHS; idx += kThreads) {
          const int rr = idx / RHS, r = idx % RHS;
          if (rr > c && rr < nr && r < nrhs) s_y[rr][r] -= s_d[rr][c] * s_y[c][r];
        }
        __syncthreads();
      }
    } else {
      for (int c = nr - 1; c >= 0; --c) {
        if (tid < nrhs) s_y[c][tid] = s_y[c][tid] / s_d[c][c];
        __syncthreads();
        for (int idx = tid; idx < kBs * RHS; idx += kThreads) {
          const int rr = idx / RHS, r = idx % RHS;
          if (rr < c && r < nrhs) s_y[rr][r] -= s_d[rr][c] * s_y[c][r];
        }
        __syncthreads();
      }
    }
    for (int idx = tid; idx < kBs * RHS; idx += kThreads) {
      const int rr = idx / RHS, r = idx % RHS;
      if (rr < nr && r < nrhs) Y[(size_t)r * ldy + r0 + rr] = s_y[rr][r];
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      st_release_u32(flags + blk, epoch);
    }
  }
}

__global__ void k_check_finite(const double* __restrict__ X, long ldx, int n, int nrhs, int* status) {
  const long total = (long)n * nrhs;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
    const long r = idx / n, i = idx % n;
    if (!isfinite(X[r * ldx + i])) {
      atomicExch(status, (int)kNotFinite);
      return;
    }
  }
}

struct TrsvScratch {
  // [ticket (256 B)] [flags nblk unsigned, rounded] [Y n x kMaxRhs doubles]
  static size_t flags_off() { return 256; }
  static size_t y_off(int n) { return (256 + (size_t)((n + kBs - 1) / kBs) * 4 + 255) / 256 * 256; }
  static size_t bytes(int n) { return y_off(n) + (size_t)n * kMaxRhs * sizeof(double); }
};

// Epochs of the readiness flags, shared by every solve of the process (any thread): each solve takes
// two consecutive values, never 0 (the flags' initial value).
std::atomic<unsigned> g_epoch{0};
unsigned next_epochs() {
  unsigned e;
  do {
    e = g_epoch.fetch_add(2) + 2;
  } while (e == 0);
  return e;
}

}  // namespace

cudaError_t lu_perm_from_ipiv(const int* ipiv, int n, int* perm, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_perm_init<<<(n + 255) / 256, 256, 0, s>>>(perm, n); BGPU_COUNT_LAUNCH();
  k_perm_compose<<<1, 1024, 0, s>>>(ipiv, n, perm); BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

size_t trsv_scratch_bytes(int n);  // (below: the base scratch and the split solves' area)

// Solves in place with FP64 factors.  The scratch must hold trsv_scratch_bytes(n) bytes and be
// zeroed once when first allocated (the flags carry an epoch; no per-call clearing is needed).
cudaError_t getrs64(const double* LU, long lda, int n, const int* perm, double* X, long ldx, int nrhs, void* scratch,
                    int* d_status, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return cudaSuccess;
  if (nrhs > kMaxRhs) return cudaErrorInvalidValue;
  unsigned char* base = static_cast<unsigned char*>(scratch);
  unsigned* ticket = reinterpret_cast<unsigned*>(base);
  unsigned* flags = reinterpret_cast<unsigned*>(base + TrsvScratch::flags_off());
  double* Y = reinterpret_cast<double*>(base + TrsvScratch::y_off(n));
  const long ldy = n;
  k_gather_rows<double><<<(n + 255) / 256, 256, 0, s>>>(X, ldx, perm, n, nrhs, Y, ldy); BGPU_COUNT_LAUNCH();
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int nblk = (n + kBs - 1) / kBs;
  const int grid = std::min(nblk, sms * 2);
  const unsigned epoch = next_epochs();
  cudaError_t e = cudaMemsetAsync(ticket, 0, 4, s);
  if (e != cudaSuccess) return e;
  BGPU_COUNT_LAUNCH();
  if (nrhs <= 8)
    k_trsv<double, true, 8><<<grid, kThreads, 0, s>>>(LU, lda, n, Y, ldy, nrhs, flags, ticket, epoch, d_status);
  else
    k_trsv<double, true, 16><<<grid, kThreads, 0, s>>>(LU, lda, n, Y, ldy, nrhs, flags, ticket, epoch, d_status);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(ticket, 0, 4, s)) != cudaSuccess) return e;
  BGPU_COUNT_LAUNCH();
  if (nrhs <= 8)
    k_trsv<double, false, 8><<<grid, kThreads, 0, s>>>(LU, lda, n, Y, ldy, nrhs, flags, ticket, epoch + 1, d_status);
  else
    k_trsv<double, false, 16><<<grid, kThreads, 0, s>>>(LU, lda, n, Y, ldy, nrhs, flags, ticket, epoch + 1,
                                                         d_status);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_copy_cols<double><<<(n + 255) / 256, 256, 0, s>>>(Y, ldy, n, nrhs, X, ldx); BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

namespace {

// ---------------------------------------------------------------------------------------------
// Triangular solves with inverted diagonal blocks (128 rows): the in-block step is a 128 x 128
// mat-vec instead of a 128-step substitution, which shortens the block-to-block dependency chain.
// ---------------------------------------------------------------------------------------------
constexpr int kIb = 128;  // rows per block
constexpr int kIrhs = 8;  // right-hand sides per pass

// Inverses of the 128 x 128 diagonal blocks of an LU factor (F = double or float): block b of DL is
// L_bb^-1 (unit lower), of DU U_bb^-1, column-major 128 x 128 (the last block padded with zeros);
// one CTA per block, one thread per column, FP64 arithmetic.
template <typename F, typename FI>
__global__ void __launch_bounds__(kIb) k_diag_inverses(const F* __restrict__ LU, long lda, int n, int b0,
                                                       FI* __restrict__ DL, FI* __restrict__ DU) {
  extern __shared__ double sdi[];  // sdi[c * (kIb + 1) + r] = factor entry (r, c) of the block
  const int b = b0 + blockIdx.x, r0 = b * kIb, h = min(kIb, n - r0), c = threadIdx.x;
  auto sl = [&](int col, int r) -> double { return sdi[col * (kIb + 1) + r]; };
  for (int i = 0; i < h; ++i)
    if (c < h) sdi[c * (kIb + 1) + i] = (double)LU[(size_t)(r0 + c) * lda + r0 + i];
  __syncthreads();
  FI* dl = DL + (size_t)b * kIb * kIb;
  FI* du = DU + (size_t)b * kIb * kIb;
  // column c of L^-1: x_c = 1, x_i = -sum_{c <= j < i} L_ij x_j  (i > c); and of U^-1:
  // x_c = 1/U_cc, x_i = -(sum_{i < j <= c} U_ij x_j) / U_ii (i < c)
  double x[kIb];
  for (int i = 0; i < kIb; ++i) x[i] = 0.0;
  if (c < h) {
    x[c] = 1.0;
    for (int i = c + 1; i < h; ++i) {
      double s0 = 0.0, s1 = 0.0;
      int j = c;
      for (; j + 1 < i; j += 2) {
        s0 += sl(j, i) * x[j];
        s1 += sl(j + 1, i) * x[j + 1];
      }
      if (j < i) s0 += sl(j, i) * x[j];
      x[i] = -(s0 + s1);
    }
  }
  for (int i = 0; i < kIb; ++i) dl[(size_t)c * kIb + i] = (FI)((c < h && i < h) ? x[i] : 0.0);
  for (int i = 0; i < kIb; ++i) x[i] = 0.0;
  if (c < h) {
    x[c] = 1.0 / sl(c, c);
    for (int i = c - 1; i >= 0; --i) {
      double s0 = 0.0, s1 = 0.0;
      int j = i + 1;
      for (; j + 1 <= c; j += 2) {
        s0 += sl(j, i) * x[j];
        s1 += sl(j + 1, i) * x[j + 1];
      }
      if (j <= c) s0 += sl(j, i) * x[j];
      x[i] = -(s0 + s1) / sl(i, i);
    }
  }
  for (int i = 0; i < kIb; ++i) du[(size_t)c * kIb + i] = (FI)((c < h && i < h) ? x[i] : 0.0);
}

// One triangle on Y (n x nrhs <= kIrhs, ldy) with the block inverses DI: LOWER = unit lower L, block
// rows in increasing order; otherwise upper U, decreasing.  TRANS: the triangle is the transpose of
// the stored one (U^T, lower, with DI = DU; or L^T, upper, with DI = DL): entry (i, j) is read from
// LU(j, i) and the block inverses are applied transposed.
//
// Work is split in tasks taken in ticket order by persistent CTAs.  In the order of the solve
// (q-space: q = block row for LOWER, nblk-1-block row otherwise), row i's final task F(i) does its
// last kLead off-diagonal blocks [i - kLead, i), adds the partial sums of the blocks before them in a
// fixed order (so results do not depend on scheduling), applies the inverted diagonal block and
// publishes x_i.  The blocks before are cut, walking away from the diagonal, into chunks of 2, 4,
// 8 and then kChunk blocks, each a partial task P(i, s) that streams its blocks into a slot of its
// own and releases that slot's flag.  A chunk is issued right after the final task of its newest
// block row (the last x it needs):
// the chunks near the diagonal, which become ready last, are short, so they finish within the few
// rows the chain advances meanwhile, and the far ones, ready long before, stream the bulk of the
// factor.  The host builds the task list (every task after all tasks it waits for, so the waits
// always end; each is bounded anyway) and CTAs take it in ticket order.
constexpr int kChunk = 16;
constexpr int kLead = 2;
constexpr int kRing = 3;  // stages of the FP32 partial tasks' factor ring (32 KB each)

// D += A B on the tensor cores (mma.sync m16n8k8, TF32 operands, FP32 accumulators).  Fragments:
// lane = 4 g + t; A (16 x 8): a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4); B (8 x 8):
// b0 (t, g), b1 (t + 4, g); D (16 x 8): d0 (g, 2t), d1 (g, 2t + 1), d2 (g + 8, 2t), d3 (g + 8, 2t + 1).
__device__ __forceinline__ void mma_tf32(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// x rounded to TF32 (nearest, ties away), as the bits of an FP32 value
__device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// bytes (a multiple of 16, from a 16-byte aligned address) fetched into L2 ahead of their use
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// The chain weights' layout: a 128 x 128 block M in FP16, scaled by its largest magnitude, in the
// order the chain's tensor-core products read it: warp w (rows 16 w .. +15) and k-step s (columns
// 8 s .. +7) give lane l the A fragment (a0, a1, a2, a3) of M's 16 x 8 tile, two k-steps per 16
// bytes, so each lane loads its fragments of a block with eight 16-byte reads.  Half index of M(r, k):
__device__ __forceinline__ int chain_frag_off(int r, int k) {
  const int w = r >> 4, g = r & 7, rhi = (r >> 3) & 1, s = k >> 3, t = k & 3, khi = (k >> 2) & 1;
  return (((w * 8 + (s >> 1)) * 32 + g * 4 + t) * 2 + (s & 1)) * 4 + rhi + 2 * khi;
}
constexpr int kChainBlockHalves = kIb * kIb;  // 16,384 halves (32 KB) per block

// A triangle's chain data (one buffer per triangle, offsets in floats), all blocks in the fragment
// order above, FP16, each row scaled by its largest magnitude (128 row scales per block):
//   [0, kLags * nblk * 8192)       the weights D_b^-1 L_{b,b-l} (or D_b^-1 U_{b,b+l}) of the lags
//                                  l = 1 .. kLags: block ((l-1) nblk + b) at that many 16,384 halves
//                                  (l = 1: the chain's W_b; 2: its V_b; 3 .. 5: the final tasks')
//   wscale_off: [+ kLags nblk 128) their row scales, block ((l-1) nblk + b) at that many 128 floats
//   bscale_off: [+ nb2 * 128)      the row scales of the off-diagonal blocks
//   blocks_off: [+ nb2 * 8192)     the off-diagonal blocks of the triangle in the order of the solve:
//                                  block (i, q), q < i in q-space (q-row i is block row i of L, or
//                                  nblk-1-i of U; q-column q likewise), number i (i-1) / 2 + q
constexpr int kLags = 5;
struct ChainLayout {
  __host__ __device__ static size_t nb2(int nblk) { return (size_t)nblk * (nblk - 1) / 2; }
  __host__ __device__ static size_t wscale_off(int nblk) { return (size_t)kLags * nblk * kChainBlockHalves / 2; }
  __host__ __device__ static size_t bscale_off(int nblk) { return wscale_off(nblk) + (size_t)kLags * nblk * kIb; }
  __host__ __device__ static size_t blocks_off(int nblk) { return (bscale_off(nblk) + nb2(nblk) * kIb + 63) / 64 * 64; }
  __host__ __device__ static size_t elems(int nblk) { return blocks_off(nblk) + nb2(nblk) * kChainBlockHalves / 2; }
};

// The chain of the FP32 preconditioner (one CTA of k_trsv_inv, all 256 threads; see there):
//     x_i = c_i - W_i x_{i-1} - V_i x_{i-2}
// over the chain steps i = 0 .. nblk-1 (block row i, or nblk-1-i for the upper triangle).  Warp w
// owns rows 16 w .. +15 of every step: both products on the tensor cores (W_i x_{i-1} for x_i, and
// V_{i+1} x_{i-1} for the next step, sharing x_{i-1}'s fragments; x rounded to TF32, the weights
// carrying FP16 rounding with a scale per row).  The chain has its SM to itself (k_trsv_inv).  The
// weights of the next step are
// loaded into registers while the current step runs; c_i (entries tagged with the solve's epoch by
// the final tasks) is loaded a step ahead and taken entry by entry once its tags match, so a step
// waits on no flag.  x_{i-1}, x_i live in a ring of three 128 x 8 buffers; one barrier per step,
// after which thread 0 releases flags[block] for the tasks that need x_i.  Wt: chain_weights32's
// output for this triangle; cslot: the tagged c slots [nblk][128][8].
template <bool LOWER>
__device__ void chain_run(const float* __restrict__ Wt, int n, int nblk, float* Y, long ldy, int nrhs, unsigned* flags,
                          unsigned epoch, int* status, const unsigned long long* cslot, unsigned long long* xt,
                          float* xb0, float* xb1, float* xb2) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const __half* Wh = reinterpret_cast<const __half*>(Wt);
  const __half* Vh = Wh + (size_t)nblk * kChainBlockHalves;
  const float* scales = Wt + ChainLayout::wscale_off(nblk);  // row scales: W's [nblk][128], then V's
  auto bl = [&](int ii) { return LOWER ? ii : nblk - 1 - ii; };
  auto xbuf = [&](int k) { return k == 0 ? xb0 : (k == 1 ? xb1 : xb2); };
  uint4 aw[8], av[8];  // this lane's fragments of W_i and V_{i+1} (FP16, two k-steps per uint4)
  auto load_frags = [&](uint4 (&a)[8], const __half* base, int ii) {
    const uint4* p = reinterpret_cast<const uint4*>(base + (size_t)bl(ii) * kChainBlockHalves) + warp * 256 + lane;
#pragma unroll
    for (int m = 0; m < 8; ++m) a[m] = __ldg(p + m * 32);
  };
  const int ra = 16 * warp + g, rb = ra + 8, n0 = 2 * t;
  unsigned long long cv[4];
  auto load_c = [&](int ii) {
    const unsigned long long* p = cslot + (size_t)ii * kIb * kIrhs;
    cv[0] = ld_relaxed_u64(p + ra * kIrhs + n0);
    cv[1] = ld_relaxed_u64(p + ra * kIrhs + n0 + 1);
    cv[2] = ld_relaxed_u64(p + rb * kIrhs + n0);
    cv[3] = ld_relaxed_u64(p + rb * kIrhs + n0 + 1);
  };
  for (int e = tid; e < kIb * kIrhs; e += 256) xb2[e] = 0.f;  // x_{-1}
  // row scales of this lane's rows ra, rb: W_i's (swa, swb) and V_{i+1}'s (sva, svb)
  auto wsc = [&](int ii, int r) { return scales[(size_t)bl(ii) * kIb + r]; };
  auto vsc = [&](int ii, int r) { return scales[((size_t)nblk + bl(ii)) * kIb + r]; };
  load_frags(aw, Wh, 0);
  float swa = wsc(0, ra), swb = wsc(0, rb), sva = 0.f, svb = 0.f;
  if (nblk > 1) {
    load_frags(av, Vh, 1);
    sva = vsc(1, ra);
    svb = vsc(1, rb);
  }
  load_c(0);
  if (tid == 0) {
    for (int ii = 1; ii < 4 && ii < nblk; ++ii) prefetch_l2(Wh + (size_t)bl(ii) * kChainBlockHalves, kChainBlockHalves * 2);
    for (int ii = 2; ii < 5 && ii < nblk; ++ii) prefetch_l2(Vh + (size_t)bl(ii) * kChainBlockHalves, kChainBlockHalves * 2);
  }
  float pc[4] = {0.f, 0.f, 0.f, 0.f};  // sv_i V_i x_{i-2}, this lane's D fragment
  __syncthreads();
  for (int i = 0; i < nblk; ++i) {
    const int blk = bl(i), r0 = blk * kIb, nr = min(kIb, n - r0);
    const float* xp = xbuf((i + 2) % 3);  // x_{i-1}
    // two independent accumulators per product (the two k-steps of a 16-byte fragment load into
    // m & 1)
    float dw[2][4], dv[2][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int j = 0; j < 4; ++j) dw[a][j] = dv[a][j] = 0.f;
#pragma unroll
    for (int m = 0; m < 8; ++m)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = 16 * m + 8 * h + t;
        const unsigned h0 = to_tf32(xp[k * kIrhs + g]), h1 = to_tf32(xp[(k + 4) * kIrhs + g]);
        const unsigned pw0 = h ? aw[m].z : aw[m].x, pw1 = h ? aw[m].w : aw[m].y;
        const unsigned pv0 = h ? av[m].z : av[m].x, pv1 = h ? av[m].w : av[m].y;
        const float2 w01 = __half22float2(*reinterpret_cast<const __half2*>(&pw0));
        const float2 w23 = __half22float2(*reinterpret_cast<const __half2*>(&pw1));
        const float2 v01 = __half22float2(*reinterpret_cast<const __half2*>(&pv0));
        const float2 v23 = __half22float2(*reinterpret_cast<const __half2*>(&pv1));
        const int a = m & 1;
        mma_tf32(dw[a], __float_as_uint(w01.x), __float_as_uint(w01.y), __float_as_uint(w23.x), __float_as_uint(w23.y),
                 h0, h1);
        mma_tf32(dv[a], __float_as_uint(v01.x), __float_as_uint(v01.y), __float_as_uint(v23.x), __float_as_uint(v23.y),
                 h0, h1);
      }
    float pw[4], pv[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      pw[j] = dw[0][j] + dw[1][j];
      pv[j] = dv[0][j] + dv[1][j];
    }
    const float swa_i = swa, swb_i = swb, sva_n = sva, svb_n = svb;
    // the next step's weights, into the registers just read
    if (i + 1 < nblk) {
      load_frags(aw, Wh, i + 1);
      swa = wsc(i + 1, ra);
      swb = wsc(i + 1, rb);
    }
    if (i + 2 < nblk) {
      load_frags(av, Vh, i + 2);
      sva = vsc(i + 2, ra);
      svb = vsc(i + 2, rb);
    }
    // c_i: every entry must carry this solve's epoch (reloaded until it does, bounded)
    int fail = 0;
    {
      const unsigned long long* p = cslot + (size_t)i * kIb * kIrhs;
      unsigned spins = 0;
      while (!((unsigned)(cv[0] >> 32) == epoch && (unsigned)(cv[1] >> 32) == epoch &&
               (unsigned)(cv[2] >> 32) == epoch && (unsigned)(cv[3] >> 32) == epoch)) {
        if (++spins > c_spin_limit) {
          fail = 1;
          break;
        }
        __nanosleep(32);
        cv[0] = ld_relaxed_u64(p + ra * kIrhs + n0);
        cv[1] = ld_relaxed_u64(p + ra * kIrhs + n0 + 1);
        cv[2] = ld_relaxed_u64(p + rb * kIrhs + n0);
        cv[3] = ld_relaxed_u64(p + rb * kIrhs + n0 + 1);
      }
    }
    float x[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = __uint_as_float((unsigned)cv[j]) - pc[j] - (j < 2 ? swa_i : swb_i) * pw[j];
    float* xo = xbuf(i % 3);
    *reinterpret_cast<float2*>(xo + ra * kIrhs + n0) = make_float2(x[0], x[1]);
    *reinterpret_cast<float2*>(xo + rb * kIrhs + n0) = make_float2(x[2], x[3]);
    if (ra < nr) {
      if (n0 < nrhs) Y[(size_t)n0 * ldy + r0 + ra] = x[0];
      if (n0 + 1 < nrhs) Y[(size_t)(n0 + 1) * ldy + r0 + ra] = x[1];
    }
    if (rb < nr) {
      if (n0 < nrhs) Y[(size_t)n0 * ldy + r0 + rb] = x[2];
      if (n0 + 1 < nrhs) Y[(size_t)(n0 + 1) * ldy + r0 + rb] = x[3];
    }
    {
      // the tagged copy the tasks read (every entry of the block, zeros included)
      unsigned long long* xq = xt + (size_t)blk * kIb * kIrhs;
      const unsigned long long tag = (unsigned long long)epoch << 32;
      st_relaxed_u64(xq + ra * kIrhs + n0, tag | __float_as_uint(x[0]));
      st_relaxed_u64(xq + ra * kIrhs + n0 + 1, tag | __float_as_uint(x[1]));
      st_relaxed_u64(xq + rb * kIrhs + n0, tag | __float_as_uint(x[2]));
      st_relaxed_u64(xq + rb * kIrhs + n0 + 1, tag | __float_as_uint(x[3]));
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) pc[j] = (j < 2 ? sva_n : svb_n) * pv[j];
    if (i + 1 < nblk) load_c(i + 1);
    // x_i complete in shared memory, in Y and in the tagged copy; x_{i-1}'s buffer free for x_{i+2}
    if (__syncthreads_or(fail)) {
      if (tid == 0) atomicExch(status, (int)kWaitTimeout);
      return;
    }
    if (tid == 0) {
      // the flag is a hint (the tasks check the tags of what they read), so no fence
      st_relaxed_u32(flags + blk, epoch);
      // the weights four steps ahead into L2 (each is read once per sweep, from HBM otherwise)
      if (i + 4 < nblk) prefetch_l2(Wh + (size_t)bl(i + 4) * kChainBlockHalves, kChainBlockHalves * 2);
      if (i + 5 < nblk) prefetch_l2(Vh + (size_t)bl(i + 5) * kChainBlockHalves, kChainBlockHalves * 2);
    }
  }
}

// This lane's product of a 128 x 128 FP16 block (fragments fr, chain_frag_off order) with x
// (128 x 8, row-major in shared memory), x rounded to TF32 (the block itself carries FP16 rounding):
// d = M x (unscaled).  Four independent accumulators (k-step s into s & 3).
__device__ __forceinline__ void block_mma(const uint4 (&fr)[8], const float* xs, float (&d)[4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float da[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int j = 0; j < 4; ++j) da[a][j] = 0.f;
#pragma unroll
  for (int m = 0; m < 8; ++m)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = 16 * m + 8 * h + t;
      const unsigned h0 = to_tf32(xs[k * kIrhs + g]), h1 = to_tf32(xs[(k + 4) * kIrhs + g]);
      const unsigned p0 = h ? fr[m].z : fr[m].x, p1 = h ? fr[m].w : fr[m].y;
      const float2 a01 = __half22float2(*reinterpret_cast<const __half2*>(&p0));
      const float2 a23 = __half22float2(*reinterpret_cast<const __half2*>(&p1));
      mma_tf32(da[(2 * m + h) & 3], __float_as_uint(a01.x), __float_as_uint(a01.y), __float_as_uint(a23.x),
               __float_as_uint(a23.y), h0, h1);
    }
#pragma unroll
  for (int j = 0; j < 4; ++j) d[j] = (da[0][j] + da[1][j]) + (da[2][j] + da[3][j]);
}

// The tasks of the FP32 preconditioner's chained triangle, run by every CTA but the chain's (the
// task list and its order as in k_trsv_inv).  The off-diagonal blocks come from the triangle's FP16
// copy (ChainLayout, k_pblocks32) and are multiplied on the tensor cores, x rounded to TF32.  Warp w,
// lane 4 g + t owns rows ra = 16 w + g and rb = ra + 8, right-hand sides 2t and 2t + 1 of its block
// row (the D fragment).
//   partial task: its blocks stream through a ring of kRing 32 KB stages (asynchronous copies
//     issued kRing - 1 blocks ahead, evict-first); each block's x goes to shared memory once its
//     flag is set; the sum into the task's slot, then the slot's flag.
//   final task: b and the slots (far ones first; the nearest covers blocks up to i-6, so all are in
//     before the final blocks' x), e = D_i^-1 (b - sum) with three TF32 products per k-step (D and
//     the sum both split: FP32-accurate), then c_i = e - sum_{l=3..5} (D_i^-1 L_{i,i-l}) x_{i-l}
//     through the lag weights (chain_weights32), each term as soon as its x is set: after x_{i-3}
//     only one 128 x 128 x 8 product remains.  c_i goes to the c slot, each entry tagged with the
//     solve's epoch.
// s_x, s_y2: 128 x 8 floats each; s_dyn: kRing x 32 KB (the ring, or D^-1 with column stride 136).
template <bool LOWER>
__device__ void chain_tasks(const float* __restrict__ Wt, const float* __restrict__ DI, int n, int nblk,
                            const float* Y, long ldy, int nrhs, const unsigned* flags, unsigned* ticket,
                            unsigned epoch, int* status, unsigned* pflags, float* part, int smax,
                            const int4* __restrict__ tasks, int ntasks, unsigned long long* cslot,
                            const unsigned long long* xt, unsigned char* s_dyn, float* s_x, float* s_y2, int* s_task,
                            int* s_cnt) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const int ra = 16 * warp + g, rb = ra + 8, n0 = 2 * t;
  const __half* blocks = reinterpret_cast<const __half*>(Wt + ChainLayout::blocks_off(nblk));
  const float* bscale = Wt + ChainLayout::bscale_off(nblk);
  const unsigned long long pol = l2_evict_first();  // the factor and D^-1 are read once per sweep
  // x of block jb from the chain's tagged copy into this thread's four entries of the 128 x 8
  // row-major tile; true when all four carry this solve's epoch
  auto fetch_x = [&](int jb, float (&xr)[4]) {
    const unsigned long long* p = xt + (size_t)jb * kIb * kIrhs + tid;
    bool ok = true;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const unsigned long long v = ld_relaxed_u64(p + 256 * e);
      ok = ok && (unsigned)(v >> 32) == epoch;
      xr[e] = __uint_as_float((unsigned)v);
    }
    return ok;
  };
  // every thread's entries valid (refetched until they are, bounded); a barrier of the whole CTA
  auto settle_x = [&](int jb, float (&xr)[4], bool ok) {
    unsigned spins = 0;
    while (!__syncthreads_and(ok)) {
      if (++spins > c_spin_limit) {
        if (tid == 0) atomicExch(status, (int)kWaitTimeout);
        return false;
      }
      __nanosleep(64);
      if (!ok) ok = fetch_x(jb, xr);
    }
    return true;
  };
  auto wait_x = [&](int jb, int blk) {
    return LOWER ? wait_ready(flags, jb, +1, 0, blk, epoch, status, s_cnt)
                 : wait_ready(flags, jb, -1, blk + 1, nblk, epoch, status, s_cnt);
  };
  for (;;) {
    if (tid == 0) {
      const unsigned tk_ = atomicAdd(ticket, 1u);
      const int4 tk = tk_ < (unsigned)ntasks ? tasks[tk_] : make_int4(0, -1, 0, 0);
      s_task[0] = tk.x;
      s_task[1] = tk.y;
      s_task[2] = tk.z;
      s_task[3] = tk.w;
    }
    __syncthreads();
    const int code = s_task[0], i = s_task[1], q0 = s_task[2], q1 = s_task[3];
    if (i < 0) return;
    const int blk = LOWER ? i : nblk - 1 - i;
    const int r0 = blk * kIb, nr = min(kIb, n - r0);
    const size_t tri = (size_t)i * (i - 1) / 2;  // the first block of q-row i in the copy
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    if (code >= 0) {
      // partial task: blocks [q0, q1) through the ring (stage st = block q0 + st)
      const int nst = q1 - q0;
      uint4* ring = reinterpret_cast<uint4*>(s_dyn);
      auto issue = [&](int st) {
        if (st < nst) {
          const uint4* src = reinterpret_cast<const uint4*>(blocks + (tri + q0 + st) * kChainBlockHalves);
          uint4* dst = ring + (st % kRing) * (kChainBlockHalves / 8);
          for (int e = tid; e < kChainBlockHalves / 8; e += 256) cp_async16z(dst + e, src + e, 16, pol);
        }
        cp_async_commit();
      };
#pragma unroll
      for (int st = 0; st < kRing - 1; ++st) issue(st);
      int confirmed = q0;
      bool have_x = false, xok = false;  // xr already holds the x of block q0 + st (all valid: xok)
      float xr[4];
      for (int st = 0; st < nst; ++st) {
        const int q = q0 + st, jb = LOWER ? q : nblk - 1 - q;
        if (q >= confirmed) {
          const int c = wait_x(jb, blk);
          if (c == 0) {
            cp_async_wait_all();
            return;
          }
          confirmed = q + c;
        }
        if (!have_x) xok = fetch_x(jb, xr);
        cp_async_wait_group<kRing - 2>();
        // x valid everywhere and stage st in for every thread; nobody reads the previous stage or x
        // any more
        if (!settle_x(jb, xr, xok)) {
          cp_async_wait_all();
          return;
        }
        issue(st + kRing - 1);
#pragma unroll
        for (int e = 0; e < 4; ++e) s_x[tid + 256 * e] = xr[e];
        __syncthreads();
        have_x = q + 1 < q1 && q + 1 < confirmed;
        if (have_x) xok = fetch_x(LOWER ? q + 1 : nblk - 2 - q, xr);  // the next block's x, its flag seen
        uint4 fr[8];
        const uint4* sp = ring + (st % kRing) * (kChainBlockHalves / 8) + warp * 256 + lane;
#pragma unroll
        for (int m = 0; m < 8; ++m) fr[m] = sp[m * 32];
        float d[4];
        block_mma(fr, s_x, d);
        const float sca = bscale[(tri + q) * kIb + ra], scb = bscale[(tri + q) * kIb + rb];
        acc[0] -= sca * d[0];
        acc[1] -= sca * d[1];
        acc[2] -= scb * d[2];
        acc[3] -= scb * d[3];
      }
      float* slot = part + ((size_t)i * smax + code) * kIb * kIrhs;
      *reinterpret_cast<float2*>(slot + ra * kIrhs + n0) = make_float2(acc[0], acc[1]);
      *reinterpret_cast<float2*>(slot + rb * kIrhs + n0) = make_float2(acc[2], acc[3]);
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        st_release_u32(pflags + (size_t)i * smax + code, epoch);
      }
      continue;
    }
    // final task.  Before any wait: D^-1 into shared memory (column stride 136), b, and the first
    // lag weight's fragments
    float* sd = reinterpret_cast<float*>(s_dyn);
    {
      const float* dblk = DI + (size_t)blk * kIb * kIb;
      for (int e = tid; e < kIb * kIb / 4; e += 256) {
        const int c = e >> 5, r4 = (e & 31) * 4;
        cp_async16z(sd + c * 136 + r4, dblk + c * kIb + r4, 16, pol);
      }
      cp_async_commit();
    }
    acc[0] = (ra < nr && n0 < nrhs) ? Y[(size_t)n0 * ldy + r0 + ra] : 0.f;
    acc[1] = (ra < nr && n0 + 1 < nrhs) ? Y[(size_t)(n0 + 1) * ldy + r0 + ra] : 0.f;
    acc[2] = (rb < nr && n0 < nrhs) ? Y[(size_t)n0 * ldy + r0 + rb] : 0.f;
    acc[3] = (rb < nr && n0 + 1 < nrhs) ? Y[(size_t)(n0 + 1) * ldy + r0 + rb] : 0.f;
    // the weight D_i^-1 L_{i,q} of q-block q (lag i - q) of this block row: fragments and row scales
    uint4 fr[8];
    float swa = 0.f, swb = 0.f;
    auto load_weight = [&](int q) {
      const size_t wb = (size_t)(i - q - 1) * nblk + blk;
      const uint4* p = reinterpret_cast<const uint4*>(reinterpret_cast<const __half*>(Wt) + wb * kChainBlockHalves) +
                       warp * 256 + lane;
#pragma unroll
      for (int m = 0; m < 8; ++m) fr[m] = __ldg(p + m * 32);
      swa = Wt[ChainLayout::wscale_off(nblk) + wb * kIb + ra];
      swb = Wt[ChainLayout::wscale_off(nblk) + wb * kIb + rb];
    };
    if (q0 < q1) load_weight(q0);
    // the slots: [2, nparts) in batches of up to eight from the top, each added once all its slots
    // are in, then slot 1 and slot 0 (all ready before the final blocks' x).  The order of the sum is
    // fixed.
    const int nparts = -1 - code;
    const unsigned* pf = pflags + (size_t)i * smax;
    const float* ps = part + (size_t)i * smax * kIb * kIrhs;
    for (int hi = nparts; hi > 2; hi -= 8) {
      const int lo = max(2, hi - 8);
      if (!wait_all(pf, lo, hi, epoch, status, s_cnt)) {
        cp_async_wait_all();
        return;
      }
      float2 va[8], vb[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int sp = lo + u;
        va[u] = sp < hi ? __ldcg(reinterpret_cast<const float2*>(ps + (size_t)sp * kIb * kIrhs + ra * kIrhs + n0))
                        : make_float2(0.f, 0.f);
        vb[u] = sp < hi ? __ldcg(reinterpret_cast<const float2*>(ps + (size_t)sp * kIb * kIrhs + rb * kIrhs + n0))
                        : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        acc[0] += va[u].x;
        acc[1] += va[u].y;
        acc[2] += vb[u].x;
        acc[3] += vb[u].y;
      }
    }
    for (int sp = min(nparts, 2) - 1; sp >= 0; --sp) {
      if (!wait_all(pf, sp, sp + 1, epoch, status, s_cnt)) {
        cp_async_wait_all();
        return;
      }
      const float2 a = __ldcg(reinterpret_cast<const float2*>(ps + (size_t)sp * kIb * kIrhs + ra * kIrhs + n0));
      const float2 b = __ldcg(reinterpret_cast<const float2*>(ps + (size_t)sp * kIb * kIrhs + rb * kIrhs + n0));
      acc[0] += a.x;
      acc[1] += a.y;
      acc[2] += b.x;
      acc[3] += b.y;
    }
    // e = D^-1 (b - sum): three TF32 products per k-step (D and the sum both split: FP32-accurate),
    // four independent accumulators (k-step s into s & 3)
    *reinterpret_cast<float2*>(s_y2 + ra * kIrhs + n0) = make_float2(acc[0], acc[1]);
    *reinterpret_cast<float2*>(s_y2 + rb * kIrhs + n0) = make_float2(acc[2], acc[3]);
    cp_async_wait_all();
    __syncthreads();
    float ca[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < 4; ++j) ca[a][j] = 0.f;
#pragma unroll
    for (int s = 0; s < kIb / 8; ++s) {
      const int k = 8 * s + t;
      const float a0 = sd[k * 136 + ra], a1 = sd[k * 136 + rb], a2 = sd[(k + 4) * 136 + ra], a3 = sd[(k + 4) * 136 + rb];
      const unsigned ah0 = to_tf32(a0), ah1 = to_tf32(a1), ah2 = to_tf32(a2), ah3 = to_tf32(a3);
      const unsigned al0 = to_tf32(a0 - __uint_as_float(ah0)), al1 = to_tf32(a1 - __uint_as_float(ah1));
      const unsigned al2 = to_tf32(a2 - __uint_as_float(ah2)), al3 = to_tf32(a3 - __uint_as_float(ah3));
      const float y0 = s_y2[k * kIrhs + g], y1 = s_y2[(k + 4) * kIrhs + g];
      const unsigned yh0 = to_tf32(y0), yh1 = to_tf32(y1);
      const unsigned yl0 = to_tf32(y0 - __uint_as_float(yh0)), yl1 = to_tf32(y1 - __uint_as_float(yh1));
      mma_tf32(ca[s & 3], al0, al1, al2, al3, yh0, yh1);
      mma_tf32(ca[s & 3], ah0, ah1, ah2, ah3, yl0, yl1);
      mma_tf32(ca[s & 3], ah0, ah1, ah2, ah3, yh0, yh1);
    }
    float cc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) cc[j] = (ca[0][j] + ca[1][j]) + (ca[2][j] + ca[3][j]);
    // c_i = e - sum over the final blocks q of D_i^-1 L_{i,q} x_q, each as soon as x_q is set (the
    // next weight's fragments loaded after each product)
    for (int q = q0; q < q1; ++q) {
      const int jb = LOWER ? q : nblk - 1 - q;
      float xr[4];
      // x_q polled in the tagged copy itself (no flag); settle_x's barriers also end every read of
      // s_x and s_y2
      if (!settle_x(jb, xr, fetch_x(jb, xr))) {
        cp_async_wait_all();
        return;
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) s_x[tid + 256 * e] = xr[e];
      __syncthreads();
      float d[4];
      block_mma(fr, s_x, d);
      cc[0] -= swa * d[0];
      cc[1] -= swa * d[1];
      cc[2] -= swb * d[2];
      cc[3] -= swb * d[3];
      if (q + 1 < q1) load_weight(q + 1);
    }
    // c_i, row-major 128 x 8, zero beyond nr and nrhs, each entry tagged with the solve's epoch in
    // its upper 32 bits (the chain takes the entries once their tags match; no flag)
    unsigned long long* cp = cslot + (size_t)i * kIb * kIrhs;
    const unsigned long long tag = (unsigned long long)epoch << 32;
    st_relaxed_u64(cp + ra * kIrhs + n0, tag | __float_as_uint((ra < nr && n0 < nrhs) ? cc[0] : 0.f));
    st_relaxed_u64(cp + ra * kIrhs + n0 + 1, tag | __float_as_uint((ra < nr && n0 + 1 < nrhs) ? cc[1] : 0.f));
    st_relaxed_u64(cp + rb * kIrhs + n0, tag | __float_as_uint((rb < nr && n0 < nrhs) ? cc[2] : 0.f));
    st_relaxed_u64(cp + rb * kIrhs + n0 + 1, tag | __float_as_uint((rb < nr && n0 + 1 < nrhs) ? cc[3] : 0.f));
    // s_y2, s_x and D^-1 are read: the next task may overwrite them
    __syncthreads();
  }
}

// V is the type of the right-hand sides and of every sum (double; float for the FP32 preconditioner).
// CHAIN (the FP32 preconditioner): the chain of block rows is taken off the task list.  A final
// task of row i then stops short of block i-2: it forms c_i = D_i^-1 (b_i - sum_{j <= i-3} L_ij x_j)
// into a slot of its own (entries tagged with the solve's epoch); CTA 0 runs the chain (chain_run),
//     x_i = c_i - W_i x_{i-1} - V_i x_{i-2},   W_i = D_i^-1 L_{i,i-1},  V_i = D_i^-1 L_{i,i-2}
// (chain_weights32, once per factorisation), and releases flags[i] for the tasks that need x_i.
// A row's hand-off through global memory (final task, c_i, chain) thus has three chain steps to
// arrive in instead of two.  The other CTAs run chain_tasks (the factor's blocks from an FP16 copy,
// products on the tensor cores).  All CTAs of the grid are resident (a cooperative launch), so CTA 0
// always runs.
template <typename F, typename FI, bool LOWER, bool TRANS = false, typename V = double, bool CHAIN = false>
__global__ void __launch_bounds__(256, sizeof(F) == 4 ? 2 : 1) k_trsv_inv(const F* __restrict__ LU, long lda, const FI* __restrict__ DI, int n,
                                                  V* Y, long ldy, int nrhs, unsigned* flags, unsigned* ticket,
                                                  unsigned epoch, int* status, unsigned* __restrict__ pflags,
                                                  V* __restrict__ part, int smax, const int4* __restrict__ tasks,
                                                  int ntasks, const FI* __restrict__ W,
                                                  unsigned long long* cslot) {
  __shared__ __align__(16) V s_y[kIb][kIrhs];
  __shared__ V s_b[kIb][kIrhs];
  __shared__ V s_acc[2][kIb][kIrhs];
  __shared__ int s_task[4], s_cnt;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  FI* s_di = reinterpret_cast<FI*>(s_dyn);  // the inverted diagonal block, stride kIb + 1
  const int nblk = (n + kIb - 1) / kIb;
  const int tid = threadIdx.x, row = tid & (kIb - 1), half = tid >> 7;
  if constexpr (CHAIN) {
    // the chain's SM is left to the chain: CTA 0 publishes its SM (tagged with the epoch, after the
    // c slots) and a task CTA on the same SM leaves at once (if the tag does not show up within the
    // wait limit, the CTA simply takes tasks)
    unsigned long long* chain_sm = cslot + (size_t)nblk * kIb * kIrhs;
    unsigned long long* xt = chain_sm + 32;  // the chain's tagged copy of x, [nblk][128][8]
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;\n" : "=r"(smid));
    if (blockIdx.x != 0) {
      if (tid == 0) {
        unsigned spins = 0;
        unsigned long long v = ld_relaxed_u64(chain_sm);
        while ((unsigned)(v >> 32) != epoch && ++spins <= c_spin_limit) {
          __nanosleep(64);
          v = ld_relaxed_u64(chain_sm);
        }
        s_cnt = (unsigned)(v >> 32) == epoch && (unsigned)v == smid;
      }
      __syncthreads();
      if (s_cnt) return;
    } else if (tid == 0) {
      st_relaxed_u64(chain_sm, ((unsigned long long)epoch << 32) | smid);
    }
    if (blockIdx.x == 0) {
      chain_run<LOWER>(reinterpret_cast<const float*>(W), n, nblk, reinterpret_cast<float*>(Y), ldy, nrhs, flags, epoch,
                       status, cslot, xt, &s_acc[0][0][0], &s_acc[1][0][0], &s_y[0][0]);
    } else {
      chain_tasks<LOWER>(reinterpret_cast<const float*>(W), reinterpret_cast<const float*>(DI), n, nblk,
                         reinterpret_cast<const float*>(Y), ldy, nrhs, flags, ticket, epoch, status, pflags,
                         reinterpret_cast<float*>(part), smax, tasks, ntasks, cslot, xt, s_dyn, &s_y[0][0],
                         &s_b[0][0], s_task, &s_cnt);
    }
    return;
  }
  // The FP32 factor's partial tasks (column-major blocks, 8 right-hand sides) stream through a ring
  // of kRing stages in s_dyn, each 64 columns x 128 rows of a block (32 KB), filled by asynchronous
  // copies issued kRing - 1 stages ahead, so the factor's loads run under the waits for x and under
  // the products; other tasks hold their block in registers.
  constexpr bool kRingPath = sizeof(F) == 4 && sizeof(V) == 4 && kIrhs == 8 && !TRANS;
  const bool vec16 = lda % 4 == 0 && (reinterpret_cast<uintptr_t>(LU) & 15) == 0;
  for (;;) {
    // task: x = slot (partial task) or -1 - number of partial tasks (final task); y = row; [z, w) blocks
    if (tid == 0) {
      const unsigned t = atomicAdd(ticket, 1u);
      const int4 tk = t < (unsigned)ntasks ? tasks[t] : make_int4(0, -1, 0, 0);
      s_task[0] = tk.x;
      s_task[1] = tk.y;
      s_task[2] = tk.z;
      s_task[3] = tk.w;
    }
    __syncthreads();
    const int code = s_task[0], i = s_task[1], q0 = s_task[2], q1 = s_task[3];
    if (i < 0) return;
    const int kind = code < 0 ? 1 : 0, sidx = code;
    const bool fin = kind == 1;
    const int blk = LOWER ? i : nblk - 1 - i;
    const int r0 = blk * kIb, nr = min(kIb, n - r0);
    const bool live = row < nr;
    V acc[kIrhs];
#pragma unroll
    for (int r = 0; r < kIrhs; ++r) acc[r] = (V)0;
    // this thread's 64 entries of block (blk, block of q) (register path)
    F lv[64];
    auto load_lv = [&](int q) {
      const int jb = LOWER ? q : nblk - 1 - q;
      const int c0 = jb * kIb, nc = min(kIb, n - c0);
      if (TRANS) {
        const F* rowp = LU + (size_t)(r0 + row) * lda + c0 + half * 64;
#pragma unroll
        for (int kk = 0; kk < 64; ++kk) lv[kk] = (live && half * 64 + kk < nc) ? rowp[kk] : (F)0;
      } else {
        const F* col = LU + (size_t)(c0 + half * 64) * lda + r0 + row;
#pragma unroll
        for (int kk = 0; kk < 64; ++kk) lv[kk] = (live && half * 64 + kk < nc) ? col[(size_t)kk * lda] : (F)0;
      }
    };
    bool lv_ready = false;  // lv already holds block q0
    if (fin) {
      // before any wait: the inverted diagonal block into shared memory (asynchronous copies), the
      // block's right-hand sides, and this thread's entries of the first block
      const FI* dblk = DI + (size_t)blk * kIb * kIb;
      for (int e = tid; e < kIb * kIb; e += 256) cp_async_elem<sizeof(FI)>(s_di + (e >> 7) * (kIb + 1) + (e & 127), dblk + e);
      for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
        const int rr = idx / kIrhs, r = idx % kIrhs;
        s_b[rr][r] = (rr < nr && r < nrhs) ? Y[(size_t)r * ldy + r0 + rr] : (V)0;
      }
      if (q0 < q1) {
        load_lv(q0);
        lv_ready = true;
      }
      // the partial sums of this row, far chunks first (ready long before): slots [2, nparts) in
      // batches of up to eight from the top, each added once all of its slots are in, half 0 taking
      // a batch's even and half 1 its odd offsets; then slot 1 (half 1).  Slot 0, the chunk next to
      // the final blocks and ready last, is added after the final blocks' product.  The order of the
      // sum is fixed.
      const int nparts = -1 - code;
      const unsigned* pf = pflags + (size_t)i * smax;
      const V* p = part + (size_t)i * smax * kIb * kIrhs + (size_t)row * kIrhs;
      for (int hi = nparts; hi > 2; hi -= 8) {
        const int lo = max(2, hi - 8);
        if (!wait_all(pf, lo, hi, epoch, status, &s_cnt)) {
          cp_async_wait_all();
          return;
        }
        V t[4][kIrhs];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int sp = lo + half + 2 * u;
#pragma unroll
          for (int r = 0; r < kIrhs; ++r) t[u][r] = sp < hi ? __ldcg(p + (size_t)sp * kIb * kIrhs + r) : (V)0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int r = 0; r < kIrhs; ++r) acc[r] += t[u][r];
      }
      if (!wait_all(pf, 1, min(nparts, 2), epoch, status, &s_cnt)) {
        cp_async_wait_all();
        return;
      }
      if (nparts > 1 && half == 1)
#pragma unroll
        for (int r = 0; r < kIrhs; ++r) acc[r] += __ldcg(p + (size_t)kIb * kIrhs + r);
    }
    if constexpr (kRingPath) {
      if (!fin) {
        // stage st: columns 64 (st & 1) .. +63 of the block of q0 + st / 2, column-major 128 x 64 at
        // ring + (st % kRing) * 8192; rows beyond nr and columns beyond n zero-filled
        float* ring = reinterpret_cast<float*>(s_dyn);
        const int nst = 2 * (q1 - q0);
        const unsigned long long pol = l2_evict_first();  // the factor is read once per sweep
        auto issue = [&](int st) {
          if (st < nst) {
            const int jb = LOWER ? q0 + (st >> 1) : nblk - 1 - q0 - (st >> 1);
            const int cs = jb * kIb + (st & 1) * 64, ncs = min(64, n - cs);
            float* dst = ring + (st % kRing) * (64 * kIb);
            const float* src = reinterpret_cast<const float*>(LU);
            if (vec16) {
              for (int e = tid; e < 64 * kIb / 4; e += 256) {
                const int c = e >> 5, rr = (e & 31) * 4;
                const int ok = c < ncs ? max(0, min(4, nr - rr)) : 0;
                cp_async16z(dst + c * kIb + rr, ok ? src + (size_t)(cs + c) * lda + r0 + rr : src, ok * 4, pol);
              }
            } else {
              for (int e = tid; e < 64 * kIb; e += 256) {
                const int c = e >> 7, rr = e & 127;
                const bool ok = c < ncs && rr < nr;
                cp_async4z(dst + c * kIb + rr, ok ? src + (size_t)(cs + c) * lda + r0 + rr : src, ok ? 4 : 0, pol);
              }
            }
          }
          cp_async_commit();
        };
#pragma unroll
        for (int st = 0; st < kRing - 1; ++st) issue(st);
        int confirmed = q0;
        bool have_x = false;  // xn holds the x of the next block
        float xn[kIb * kIrhs / 256];
        for (int st = 0; st < nst; ++st) {
          const int q = q0 + (st >> 1);
          const bool head = (st & 1) == 0;
          if (head && q >= confirmed) {
            const int jb = LOWER ? q : nblk - 1 - q;
            const int c = LOWER ? wait_ready(flags, jb, +1, 0, blk, epoch, status, &s_cnt)
                                : wait_ready(flags, jb, -1, blk + 1, nblk, epoch, status, &s_cnt);
            if (c == 0) {
              cp_async_wait_all();
              return;
            }
            confirmed = q + c;
          }
          cp_async_wait_group<kRing - 2>();
          // stage st is in for every thread; nobody reads stage st - 1 (nor, at a block's head, the
          // previous block's x) any more
          __syncthreads();
          issue(st + kRing - 1);
          if (head) {
            const int jb = LOWER ? q : nblk - 1 - q;
            const int c0 = jb * kIb, nc = min(kIb, n - c0);
            if (have_x) {
#pragma unroll
              for (int e = 0; e < kIb * kIrhs / 256; ++e) {
                const int idx = tid + 256 * e;
                s_y[idx / kIrhs][idx % kIrhs] = xn[e];
              }
            } else {
              for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
                const int rr = idx / kIrhs, r = idx % kIrhs;
                s_y[rr][r] = (rr < nc && r < nrhs) ? __ldcg(&Y[(size_t)r * ldy + c0 + rr]) : 0.f;
              }
            }
            have_x = false;
            __syncthreads();
          } else if (q + 1 < q1 && q + 1 < confirmed) {
            // the next block's x (its flag already seen), to registers while this product runs
            const int jn = LOWER ? q + 1 : nblk - 2 - q;
            const int cn = jn * kIb, nn = min(kIb, n - cn);
#pragma unroll
            for (int e = 0; e < kIb * kIrhs / 256; ++e) {
              const int idx = tid + 256 * e, rr = idx / kIrhs, r = idx % kIrhs;
              xn[e] = (rr < nn && r < nrhs) ? __ldcg(&Y[(size_t)r * ldy + cn + rr]) : 0.f;
            }
            have_x = true;
          }
          // columns 32 half .. +31 of the stage against the matching 32 rows of x (two 16-byte reads
          // of the 8 right-hand sides per row)
          const float* sl = ring + (st % kRing) * (64 * kIb) + half * 32 * kIb + row;
          const float4* sy = reinterpret_cast<const float4*>(&s_y[(st & 1) * 64 + half * 32][0]);
#pragma unroll
          for (int kk = 0; kk < 32; ++kk) {
            const float l = sl[kk * kIb];
            const float4 a = sy[2 * kk], b = sy[2 * kk + 1];
            acc[0] -= l * a.x, acc[1] -= l * a.y, acc[2] -= l * a.z, acc[3] -= l * a.w;
            acc[4] -= l * b.x, acc[5] -= l * b.y, acc[6] -= l * b.z, acc[7] -= l * b.w;
          }
        }
#pragma unroll
        for (int r = 0; r < kIrhs; ++r) s_acc[half][row][r] = acc[r];
        __syncthreads();
        V* slot = part + ((size_t)i * smax + sidx) * kIb * kIrhs;
        for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
          const int rr = idx / kIrhs, r = idx % kIrhs;
          slot[idx] = s_acc[0][rr][r] + s_acc[1][rr][r];
        }
        __syncthreads();
        if (tid == 0) {
          __threadfence();
          st_release_u32(pflags + (size_t)i * smax + sidx, epoch);
        }
        continue;
      }
    }
    int confirmed = q0;
    bool have_x = false;  // s_y already holds this block's x (loaded during the previous block)
    for (int q = q0; q < q1; ++q) {
      const int jb = LOWER ? q : nblk - 1 - q;
      const int c0 = jb * kIb, nc = min(kIb, n - c0);
      // this thread's 64 entries of block (blk, jb), loaded before the wait
      if (!(lv_ready && q == q0)) load_lv(q);
      if (q >= confirmed) {
        const int c = LOWER ? wait_ready(flags, jb, +1, 0, blk, epoch, status, &s_cnt)
                            : wait_ready(flags, jb, -1, blk + 1, nblk, epoch, status, &s_cnt);
        if (c == 0) {
          cp_async_wait_all();
          return;
        }
        confirmed = q + c;
      }
      if (!have_x)
        for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
          const int rr = idx / kIrhs, r = idx % kIrhs;
          s_y[rr][r] = (rr < nc && r < nrhs) ? __ldcg(&Y[(size_t)r * ldy + c0 + rr]) : (V)0;
        }
      __syncthreads();
      // the next block's x, when its flag is already known to be set, loaded while this block's
      // product runs (to shared memory after it)
      const bool pre = q + 1 < q1 && q + 1 < confirmed;
      V xn[kIb * kIrhs / 256];
      if (pre) {
        const int jn = LOWER ? q + 1 : nblk - 2 - q;
        const int cn = jn * kIb, nn = min(kIb, n - cn);
#pragma unroll
        for (int e = 0; e < kIb * kIrhs / 256; ++e) {
          const int idx = tid + 256 * e, rr = idx / kIrhs, r = idx % kIrhs;
          xn[e] = (rr < nn && r < nrhs) ? __ldcg(&Y[(size_t)r * ldy + cn + rr]) : (V)0;
        }
      }
      if constexpr (sizeof(V) == 4 && kIrhs == 8) {
        // (FP32: the 8 right-hand sides of a row of x as two 16-byte reads)
        const float4* sy = reinterpret_cast<const float4*>(&s_y[half * 64][0]);
#pragma unroll
        for (int kk = 0; kk < 64; ++kk) {
          const V l = (V)lv[kk];
          const float4 a = sy[2 * kk], b = sy[2 * kk + 1];
          acc[0] -= l * a.x, acc[1] -= l * a.y, acc[2] -= l * a.z, acc[3] -= l * a.w;
          acc[4] -= l * b.x, acc[5] -= l * b.y, acc[6] -= l * b.z, acc[7] -= l * b.w;
        }
      } else {
#pragma unroll
        for (int kk = 0; kk < 64; ++kk) {
          const V l = (V)lv[kk];
#pragma unroll
          for (int r = 0; r < kIrhs; ++r) acc[r] -= l * s_y[half * 64 + kk][r];
        }
      }
      __syncthreads();
      if (pre) {
#pragma unroll
        for (int e = 0; e < kIb * kIrhs / 256; ++e) {
          const int idx = tid + 256 * e;
          s_y[idx / kIrhs][idx % kIrhs] = xn[e];
        }
      }
      have_x = pre;
    }
    if (fin) {
      // slot 0 (see above)
      const int nparts = -1 - code;
      if (!wait_all(pflags + (size_t)i * smax, 0, min(nparts, 1), epoch, status, &s_cnt)) {
        cp_async_wait_all();
        return;
      }
      if (nparts > 0 && half == 0)
#pragma unroll
        for (int r = 0; r < kIrhs; ++r) acc[r] += __ldcg(part + (size_t)i * smax * kIb * kIrhs + (size_t)row * kIrhs + r);
    }
#pragma unroll
    for (int r = 0; r < kIrhs; ++r) s_acc[half][row][r] = acc[r];
    __syncthreads();
    if (!fin) {
      V* slot = part + ((size_t)i * smax + sidx) * kIb * kIrhs;
      for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
        const int rr = idx / kIrhs, r = idx % kIrhs;
        slot[idx] = s_acc[0][rr][r] + s_acc[1][rr][r];
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        st_release_u32(pflags + (size_t)i * smax + sidx, epoch);
      }
      continue;
    }
    // final task: right-hand side b + (negative) off-diagonal sums, then x = D^-1 (...)
    for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
      const int rr = idx / kIrhs, r = idx % kIrhs;
      s_y[rr][r] = s_b[rr][r] + (s_acc[0][rr][r] + s_acc[1][rr][r]);
    }
    cp_async_wait_all();
    __syncthreads();
    // each half does 64 of the 128 products; D^-1 (row, c) at s_di[c * 129 + row] (transposed:
    // the other way round)
#pragma unroll
    for (int r = 0; r < kIrhs; ++r) acc[r] = (V)0;
#pragma unroll 8
    for (int kk = 0; kk < 64; ++kk) {
      const int cc = half * 64 + kk;
      const V dv = TRANS ? (V)s_di[row * (kIb + 1) + cc] : (V)s_di[cc * (kIb + 1) + row];
#pragma unroll
      for (int r = 0; r < kIrhs; ++r) acc[r] += dv * s_y[cc][r];
    }
#pragma unroll
    for (int r = 0; r < kIrhs; ++r) s_acc[half][row][r] = acc[r];
    __syncthreads();
    if constexpr (CHAIN) {
      // c_i, row-major 128 x kIrhs, zero beyond nr and nrhs, each entry tagged with the solve's epoch
      // in its upper 32 bits (the chain takes the entries once their tags match; no flag)
      unsigned long long* cp = cslot + (size_t)i * kIb * kIrhs;
      for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
        const int rr = idx / kIrhs, r = idx % kIrhs;
        const float c = (rr < nr && r < nrhs) ? (float)(s_acc[0][rr][r] + s_acc[1][rr][r]) : 0.f;
        st_relaxed_u64(cp + idx, ((unsigned long long)epoch << 32) | __float_as_uint(c));
      }
    } else {
      for (int idx = tid; idx < kIb * kIrhs; idx += 256) {
        const int rr = idx / kIrhs, r = idx % kIrhs;
        if (rr < nr && r < nrhs) Y[(size_t)r * ldy + r0 + rr] = s_acc[0][rr][r] + s_acc[1][rr][r];
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        st_release_u32(flags + blk, epoch);
      }
    }
  }
}

// The chain weights of the FP32 preconditioner (see chain_run, chain_tasks), one triangle per
// blockIdx.y, one block row b per blockIdx.x, one lag l = 1 + blockIdx.z (1 .. kLags):
//   D_b^-1 L_{b,b-l} (lower) or D_b^-1 U_{b,b+l} (upper)
// in FP16 with every row scaled by its largest magnitude, in the fragment order of chain_frag_off
// (ChainLayout).  Rows and columns beyond n zero; a missing neighbour gives zeros (scales 1).
__global__ void __launch_bounds__(256) k_chain_weights32(const float* __restrict__ LU, long lda, int n,
                                                          const float* __restrict__ DL, const float* __restrict__ DU,
                                                          float* __restrict__ WL, float* __restrict__ WU) {
  extern __shared__ __align__(16) float s_w[];
  float* sd = s_w;                  // D^-1 (r, k) at sd[k * 129 + r]
  float* sb = s_w + kIb * (kIb + 1);  // the off-diagonal block (k, c) at sb[c * 129 + k]
  __shared__ unsigned s_rmax[kIb];  // each row's largest magnitude (FP32 bits)
  const int nblk = (n + kIb - 1) / kIb, b = blockIdx.x, lower = blockIdx.y == 0, lag = 1 + blockIdx.z;
  const int nb = lower ? b - lag : b + lag;  // the neighbouring block column
  float* base = lower ? WL : WU;
  __half* out16 = reinterpret_cast<__half*>(base) + ((size_t)(lag - 1) * nblk + b) * kChainBlockHalves;
  float* scale = base + ChainLayout::wscale_off(nblk) + ((size_t)(lag - 1) * nblk + b) * kIb;
  const int tid = threadIdx.x;
  if (nb < 0 || nb >= nblk) {
    for (int e = tid; e < kChainBlockHalves; e += 256) out16[e] = __float2half_rn(0.f);
    if (tid < kIb) scale[tid] = 1.f;
    return;
  }
  if (tid < kIb) s_rmax[tid] = 0u;
  const float* D = (lower ? DL : DU) + (size_t)b * kIb * kIb;
  const int r0 = b * kIb, nr = min(kIb, n - r0), c0 = nb * kIb, nc = min(kIb, n - c0);
  for (int e = tid; e < kIb * kIb; e += 256) {
    const int r = e & (kIb - 1), c = e >> 7;
    sd[c * (kIb + 1) + r] = D[e];
    sb[c * (kIb + 1) + r] = (r < nr && c < nc) ? LU[(size_t)(c0 + c) * lda + r0 + r] : 0.f;
  }
  __syncthreads();
  // thread: rows 8 (tid & 15) .. +7, columns 8 (tid >> 4) .. +7
  const int rb = 8 * (tid & 15), cb = 8 * (tid >> 4);
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  for (int k = 0; k < kIb; ++k) {
    float a[8], bv[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = sd[k * (kIb + 1) + rb + i];
#pragma unroll
    for (int j = 0; j < 8; ++j) bv[j] = sb[(cb + j) * (kIb + 1) + k];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * bv[j];
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float m = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) m = fmaxf(m, fabsf(acc[i][j]));
    if (rb + i < nr) atomicMax(&s_rmax[rb + i], __float_as_uint(m));  // non-negative: ordered as integers
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float mx = __uint_as_float(s_rmax[rb + i]), sc = mx > 0.f ? mx : 1.f, inv = 1.f / sc;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      out16[chain_frag_off(rb + i, cb + j)] = __float2half_rn((rb + i < nr) ? acc[i][j] * inv : 0.f);
  }
  if (tid < kIb) {
    const float mx = __uint_as_float(s_rmax[tid]);
    scale[tid] = mx > 0.f ? mx : 1.f;
  }
}

// The off-diagonal blocks of both triangles of the FP32 factor LU, copied in FP16 (each row scaled
// by its largest magnitude) in the chain's fragment order (ChainLayout): block blockIdx.x of
// triangle blockIdx.y (0: L, into WL; 1: U, into WU).  Rows and columns beyond n zero; an all-zero
// row gets scale 1.
__global__ void __launch_bounds__(256) k_pblocks32(const float* __restrict__ LU, long lda, int n, float* __restrict__ WL,
                                                    float* __restrict__ WU) {
  extern __shared__ __align__(16) float s_blk[];  // element (r, k) at k * 129 + r
  __shared__ float s_rm[2][kIb], s_inv[kIb];
  const int nblk = (n + kIb - 1) / kIb, tid = threadIdx.x;
  const long idx = blockIdx.x;
  // q-row i and q-column q of the block: idx = i (i-1) / 2 + q, q < i
  int i = (int)((1.0 + sqrt(1.0 + 8.0 * (double)idx)) * 0.5);
  while ((long)i * (i - 1) / 2 > idx) --i;
  while ((long)(i + 1) * i / 2 <= idx) ++i;
  const int q = (int)(idx - (long)i * (i - 1) / 2);
  const bool lower = blockIdx.y == 0;
  const int blk = lower ? i : nblk - 1 - i, jb = lower ? q : nblk - 1 - q;
  const int r0 = blk * kIb, nr = min(kIb, n - r0), c0 = jb * kIb, nc = min(kIb, n - c0);
  for (int e = tid; e < kIb * kIb; e += 256) {
    const int r = e & (kIb - 1), k = e >> 7;
    s_blk[k * (kIb + 1) + r] = (r < nr && k < nc) ? LU[(size_t)(c0 + k) * lda + r0 + r] : 0.f;
  }
  __syncthreads();
  {
    // row r's largest magnitude: thread (r, half) over columns 64 half .. +63
    const int r = tid & (kIb - 1), h = tid >> 7;
    float m = 0.f;
    for (int k = 64 * h; k < 64 * h + 64; ++k) m = fmaxf(m, fabsf(s_blk[k * (kIb + 1) + r]));
    s_rm[h][r] = m;
  }
  __syncthreads();
  float* base = lower ? WL : WU;
  if (tid < kIb) {
    const float mx = fmaxf(s_rm[0][tid], s_rm[1][tid]), sc = mx > 0.f ? mx : 1.f;
    s_inv[tid] = 1.f / sc;
    base[ChainLayout::bscale_off(nblk) + (size_t)idx * kIb + tid] = sc;
  }
  __syncthreads();
  uint4* out = reinterpret_cast<uint4*>(base + ChainLayout::blocks_off(nblk)) + (size_t)idx * (kChainBlockHalves / 8);
  // 16-byte chunk c = halves 8c .. 8c+7: warp w, two k-steps 2m, 2m+1, lane 4g + t (chain_frag_off)
  for (int c = tid; c < kChainBlockHalves / 8; c += 256) {
    const int w = c >> 8, mm = (c >> 5) & 7, lane = c & 31, g = lane >> 2, t = lane & 3;
    unsigned u[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      __half2 h2;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int jj = 2 * p + e, s = 2 * mm + (jj >> 2), j = jj & 3;
        const int r = 16 * w + g + 8 * (j & 1), k = 8 * s + t + 4 * (j >> 1);
        const __half h = __float2half_rn(s_blk[k * (kIb + 1) + r] * s_inv[r]);
        if (e == 0) h2.x = h; else h2.y = h;
      }
      u[p] = *reinterpret_cast<unsigned*>(&h2);
    }
    out[c] = make_uint4(u[0], u[1], u[2], u[3]);
  }
}

// Scratch of the split solves, after the base scratch: the partial sums' ready flags [nblk][smax]
// (zero when allocated; a slot is ready when its flag equals the solve's epoch), the partial sums
// [nblk][smax][128][kIrhs], and the task list.
struct SplitScratch {
  static int nblk(int n) { return (n + kIb - 1) / kIb; }
  static int smax(int n) { return 4 + nblk(n) / kChunk; }
  static size_t max_tasks(int n) { return (size_t)nblk(n) * (1 + smax(n)); }
  static size_t base(int n) { return (TrsvScratch::bytes(n) + 255) / 256 * 256; }
  static size_t part_off(int n) { return base(n) + ((size_t)nblk(n) * smax(n) * 4 + 255) / 256 * 256; }
  static size_t task_off(int n) { return part_off(n) + (size_t)nblk(n) * smax(n) * kIb * kIrhs * sizeof(double); }
  // the chain's c_i slots (entries tagged with the solve's epoch; zero when allocated), the chain
  // CTA's SM (tagged likewise, in a 256-byte slot) and the chain's tagged copy of x
  static size_t cslot_off(int n) { return (task_off(n) + max_tasks(n) * sizeof(int4) + 255) / 256 * 256; }
  static size_t bytes(int n) {
    return cslot_off(n) + ((size_t)nblk(n) * kIb * kIrhs * 2 + 32) * sizeof(unsigned long long);
  }
};

// The task list of a triangle with nblk block rows (see k_trsv_inv), built once per size.  chain:
// the final task of row b takes blocks b-5 .. b-3 through the weights D_b^-1 L_{b,b-l} (see
// chain_tasks; b-2 and b-1 are the chain's), the partial tasks the blocks before b-5.
const std::vector<int4>& split_tasks(int nblk, bool chain = false) {
  static std::map<int, std::vector<int4>> cache[2];
  auto it = cache[chain].find(nblk);
  if (it != cache[chain].end()) return it->second;
  std::vector<std::vector<int4>> after(nblk);  // partial tasks issued after F(b)
  std::vector<int> nparts(nblk, 0);
  const int lead = chain ? kLags : kLead;  // blocks [i - lead, i - (chain ? 2 : 0)) in the final task
  for (int i = 0; i < nblk; ++i) {
    int e = i - lead, w = 2, sidx = 0;
    while (e > 0) {
      const int lo = std::max(0, e - w);
      after[e - 1].push_back(make_int4(sidx, i, lo, e));
      e = lo;
      w = std::min(2 * w, kChunk);
      ++sidx;
    }
    nparts[i] = sidx;
  }
  std::vector<int4> list;
  for (int b = 0; b < nblk; ++b) {
    list.push_back(make_int4(-1 - nparts[b], b, std::max(0, b - lead), chain ? std::max(0, b - 2) : b));
    for (const int4& t : after[b]) list.push_back(t);
  }
  return cache[chain].emplace(nblk, std::move(list)).first->second;
}

// One triangle of the FP32 preconditioner with the chain (k_trsv_inv, CHAIN): W the chain weights
// of this triangle (chain_weights32).
template <bool LOWER>
cudaError_t trsv_one_chain(const float* LU, long lda, const float* DI, const float* W, int n, float* Yc, long ldy,
                           int q, void* scratch, unsigned epoch, int* d_status, cudaStream_t s) {
  unsigned char* base = static_cast<unsigned char*>(scratch);
  unsigned* ticket = reinterpret_cast<unsigned*>(base);
  unsigned* flags = reinterpret_cast<unsigned*>(base + TrsvScratch::flags_off());
  unsigned* pflags = reinterpret_cast<unsigned*>(base + SplitScratch::base(n));
  float* part = reinterpret_cast<float*>(base + SplitScratch::part_off(n));
  int4* tasks = reinterpret_cast<int4*>(base + SplitScratch::task_off(n));
  unsigned long long* cslot = reinterpret_cast<unsigned long long*>(base + SplitScratch::cslot_off(n));
  const std::vector<int4>& list = split_tasks(SplitScratch::nblk(n), true);
  if (list.size() > SplitScratch::max_tasks(n)) return cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaMemsetAsync(ticket, 0, 4, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(tasks, list.data(), list.size() * sizeof(int4), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return e;
  // the final tasks' inverted diagonal block (128 x 129 FP32) or the partial tasks' ring (kRing x
  // 32 KB); the chain uses none
  const size_t dsmem = std::max((size_t)kIb * (kIb + 1) * sizeof(float), (size_t)kRing * 64 * kIb * 4);
  auto kern = k_trsv_inv<float, float, LOWER, false, float, true>;
  static bool attr = false;
  static int per_sm = 0;
  if (!attr) {
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem)) != cudaSuccess)
      return e;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, dsmem) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    per_sm = std::min(per_sm, 2);
    attr = true;
  }
  // a cooperative launch: every CTA resident (CTA 0 runs the chain the others wait on); the rest take
  // tasks in ticket order
  const float* di = DI;
  float* y = Yc;
  long ldy_ = ldy;
  int n_ = n, q_ = q, smax = SplitScratch::smax(n), nt = (int)list.size();
  unsigned ep = epoch;
  void* args[] = {(void*)&LU, (void*)&lda, (void*)&di, (void*)&n_, (void*)&y, (void*)&ldy_, (void*)&q_,
                  (void*)&flags, (void*)&ticket, (void*)&ep, (void*)&d_status, (void*)&pflags, (void*)&part,
                  (void*)&smax, (void*)&tasks, (void*)&nt, (void*)&W, (void*)&cslot};
  e = cudaLaunchCooperativeKernel((const void*)kern, dim3(sms * per_sm), dim3(256), args, dsmem, s);
  BGPU_COUNT_LAUNCH();
  return e;
}

// one triangle: ticket, counters and task list set, then the persistent launch (one CTA per SM)
template <typename F, typename FI, bool LOWER, bool TRANS, typename V = double>
cudaError_t trsv_one(const F* LU, long lda, const FI* DI, int n, V* Yc, long ldy, int q, void* scratch,
                     unsigned epoch, int* d_status, cudaStream_t s) {
  unsigned char* base = static_cast<unsigned char*>(scratch);
  unsigned* ticket = reinterpret_cast<unsigned*>(base);
  unsigned* flags = reinterpret_cast<unsigned*>(base + TrsvScratch::flags_off());
  unsigned* pflags = reinterpret_cast<unsigned*>(base + SplitScratch::base(n));
  V* part = reinterpret_cast<V*>(base + SplitScratch::part_off(n));
  int4* tasks = reinterpret_cast<int4*>(base + SplitScratch::task_off(n));
  const std::vector<int4>& list = split_tasks(SplitScratch::nblk(n));
  if (list.size() > SplitScratch::max_tasks(n)) return cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaMemsetAsync(ticket, 0, 4, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(tasks, list.data(), list.size() * sizeof(int4), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return e;
  // the final tasks' inverted diagonal block; for the FP32 factor at least the partial tasks' ring
  const size_t dsmem = std::max((size_t)kIb * (kIb + 1) * sizeof(FI),
                                sizeof(F) == 4 && !TRANS ? (size_t)kRing * 64 * kIb * 4 : (size_t)0);
  static bool attr = false;
  if (!attr) {
    if ((e = cudaFuncSetAttribute(k_trsv_inv<F, FI, LOWER, TRANS, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dsmem)) != cudaSuccess)
      return e;
    attr = true;
  }
  // as many CTAs as fit (tasks are taken in ticket order and wait only on earlier tickets, so any
  // grid size completes)
  static int per_sm = 0;
  if (!per_sm) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trsv_inv<F, FI, LOWER, TRANS, V>, 256, dsmem) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    per_sm = std::min(per_sm, 2);
  }
  k_trsv_inv<F, FI, LOWER, TRANS, V><<<sms * per_sm, 256, dsmem, s>>>(LU, lda, DI, n, Yc, ldy, q, flags, ticket, epoch, d_status,
                                                          pflags, part, SplitScratch::smax(n), tasks, (int)list.size(),
                                                          nullptr, nullptr);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

template <typename F, typename FI, typename V = double>
cudaError_t trsv_inv_pair(const F* LU, long lda, const FI* DL, const FI* DU, int n, V* Y, long ldy, int nrhs,
                          void* scratch, int* d_status, cudaStream_t s) {
  for (int c0 = 0; c0 < nrhs; c0 += kIrhs) {
    const int q = std::min(kIrhs, nrhs - c0);
    V* Yc = Y + (size_t)c0 * ldy;
    const unsigned epoch = next_epochs();
    cudaError_t e = trsv_one<F, FI, true, false, V>(LU, lda, DL, n, Yc, ldy, q, scratch, epoch, d_status, s);
    if (e != cudaSuccess) return e;
    if ((e = trsv_one<F, FI, false, false, V>(LU, lda, DU, n, Yc, ldy, q, scratch, epoch + 1, d_status, s)) !=
        cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

// Y := U^-T Y, then L^-T Y (the transposed solve, FP64 factors)
cudaError_t trsv_inv_pair_trans(const double* LU, long lda, const double* DL, const double* DU, int n, double* Y,
                                long ldy, int nrhs, void* scratch, int* d_status, cudaStream_t s) {
  for (int c0 = 0; c0 < nrhs; c0 += kIrhs) {
    const int q = std::min(kIrhs, nrhs - c0);
    double* Yc = Y + (size_t)c0 * ldy;
    const unsigned epoch = next_epochs();
    cudaError_t e = trsv_one<double, double, true, true>(LU, lda, DU, n, Yc, ldy, q, scratch, epoch, d_status, s);
    if (e != cudaSuccess) return e;
    if ((e = trsv_one<double, double, false, true>(LU, lda, DL, n, Yc, ldy, q, scratch, epoch + 1, d_status, s)) !=
        cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

// X[perm[i]] = Y[i] (the inverse of k_gather_rows)
template <typename T>
__global__ void k_scatter_rows(const T* __restrict__ Y, long ldy, const int* __restrict__ perm, int n, int nrhs,
                               T* __restrict__ X, long ldx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  for (int r = 0; r < nrhs; ++r) X[(size_t)r * ldx + p] = Y[(size_t)r * ldy + i];
}

}  // namespace

// dgetrs('T') with FP64 factors and their diagonal-block inverses: X := A^-T X (in place).
// A = P^T L U, so A^T x = b is U^T L^T (P x) = b: two transposed triangular solves, then x = P^T z.
cudaError_t getrs64_trans_inv(const double* LU, long lda, const double* DL, const double* DU, int n, const int* perm,
                              double* X, long ldx, int nrhs, void* scratch, int* d_status, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return cudaSuccess;
  if (nrhs > kMaxRhs) return cudaErrorInvalidValue;
  unsigned char* base = static_cast<unsigned char*>(scratch);
  double* Y = reinterpret_cast<double*>(base + TrsvScratch::y_off(n));
  const long ldy = n;
  k_copy_cols<double><<<(n + 255) / 256, 256, 0, s>>>(X, ldx, n, nrhs, Y, ldy);
  BGPU_COUNT_LAUNCH();
  cudaError_t e = trsv_inv_pair_trans(LU, lda, DL, DU, n, Y, ldy, nrhs, scratch, d_status, s);
  if (e != cudaSuccess) return e;
  k_scatter_rows<double><<<(n + 255) / 256, 256, 0, s>>>(Y, ldy, perm, n, nrhs, X, ldx);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

size_t trsv_scratch_bytes(int n) { return SplitScratch::bytes(n); }

size_t diag_inverse_elems(int n) { return (size_t)((n + kIb - 1) / kIb) * kIb * kIb; }

constexpr size_t kDiagInvSmem = (size_t)kIb * (kIb + 1) * sizeof(double);

cudaError_t diag_inverses64(const double* LU, long lda, int n, double* DL, double* DU, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_diag_inverses<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kDiagInvSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k_diag_inverses<double, double><<<(n + kIb - 1) / kIb, kIb, kDiagInvSmem, s>>>(LU, lda, n, 0, DL, DU);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// dgetrs('N') with FP64 factors and their diagonal-block inverses: X := A^-1 X (in place).
cudaError_t getrs64_inv(const double* LU, long lda, const double* DL, const double* DU, int n, const int* perm,
                        double* X, long ldx, int nrhs, void* scratch, int* d_status, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return cudaSuccess;
  if (nrhs > kMaxRhs) return cudaErrorInvalidValue;
  unsigned char* base = static_cast<unsigned char*>(scratch);
  double* Y = reinterpret_cast<double*>(base + TrsvScratch::y_off(n));
  const long ldy = n;
  k_gather_rows<double><<<(n + 255) / 256, 256, 0, s>>>(X, ldx, perm, n, nrhs, Y, ldy);
  BGPU_COUNT_LAUNCH();
  cudaError_t e = trsv_inv_pair<double, double>(LU, lda, DL, DU, n, Y, ldy, nrhs, scratch, d_status, s);
  if (e != cudaSuccess) return e;
  k_copy_cols<double><<<(n + 255) / 256, 256, 0, s>>>(Y, ldy, n, nrhs, X, ldx);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// Y := U^-1 L^-1 Y with FP32 factors of an unpivoted LU and their FP32 diagonal-block inverses,
// FP32 right-hand sides and sums (the preconditioner of the refined solve, whose result only
// steers the iteration: the FP64 products and residuals fix the accuracy)
cudaError_t trsv_lu32_inv(const float* LU, long lda, const float* DL, const float* DU, const float* WL,
                          const float* WU, int n, float* Y, long ldy, int nrhs, void* scratch, int* d_status,
                          cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return cudaSuccess;
  if (!WL || !WU) return trsv_inv_pair<float, float, float>(LU, lda, DL, DU, n, Y, ldy, nrhs, scratch, d_status, s);
  for (int c0 = 0; c0 < nrhs; c0 += kIrhs) {
    const int q = std::min(kIrhs, nrhs - c0);
    float* Yc = Y + (size_t)c0 * ldy;
    const unsigned epoch = next_epochs();
    cudaError_t e = trsv_one_chain<true>(LU, lda, DL, WL, n, Yc, ldy, q, scratch, epoch, d_status, s);
    if (e != cudaSuccess) return e;
    if ((e = trsv_one_chain<false>(LU, lda, DU, WU, n, Yc, ldy, q, scratch, epoch + 1, d_status, s)) != cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

cudaError_t set_wait_limit(unsigned spins) { return cudaMemcpyToSymbol(c_spin_limit, &spins, sizeof spins); }

size_t chain_weights_elems(int n) { return ChainLayout::elems((n + kIb - 1) / kIb); }

cudaError_t chain_weights32(const float* LU, long lda, const float* DL, const float* DU, int n, float* WL, float* WU,
                            cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const size_t smem = (size_t)2 * kIb * (kIb + 1) * sizeof(float);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_chain_weights32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int nblk = (n + kIb - 1) / kIb;
  k_chain_weights32<<<dim3(nblk, 2, kLags), 256, smem, s>>>(LU, lda, n, DL, DU, WL, WU);
  BGPU_COUNT_LAUNCH();
  const size_t nb2 = ChainLayout::nb2(nblk);
  if (nb2 > 0) {
    static bool attr_b = false;
    if (!attr_b) {
      cudaError_t e = cudaFuncSetAttribute(k_pblocks32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(kIb * (kIb + 1) * sizeof(float)));
      if (e != cudaSuccess) return e;
      attr_b = true;
    }
    k_pblocks32<<<dim3((unsigned)nb2, 2), 256, kIb * (kIb + 1) * sizeof(float), s>>>(LU, lda, n, WL, WU);
    BGPU_COUNT_LAUNCH();
  }
  return cudaGetLastError();
}

cudaError_t check_finite(const double* X, long ldx, int n, int nrhs, int* d_status, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return cudaSuccess;
  k_check_finite<<<std::min(1184, (n * nrhs + 255) / 256), 256, 0, s>>>(X, ldx, n, nrhs, d_status); BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// bgpu_dgetrs_noalloc: the solve without any device allocation
// ---------------------------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocBytes = sizeof(g_noalloc_scratch);
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_base[kMaxDevices] = {};

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// [0, 256) status word | trsv scratch (ticket, readiness flags, permuted right-hand sides) | perm
size_t noalloc_bytes(int n) { return 256 + round256(TrsvScratch::bytes(n)) + round256(4 * (size_t)n); }

int noalloc_max_n() {
  int lo = 0, hi = 1 << 24;
  while (lo < hi) {
    const int mid = lo + (hi - lo + 1) / 2;
    if (noalloc_bytes(mid) <= kNoAllocBytes) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Once per device, with that device current: the device address of the scratch, zeroed.
cudaError_t noalloc_base(unsigned char** out, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_base[dev]) {
    void* p = nullptr;
    if ((e = cudaGetSymbolAddress(&p, g_noalloc_scratch)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(p, 0, kNoAllocBytes, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    g_noalloc_base[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_base[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace bgpu

using bgpu::log_message;

namespace bgpu {
namespace {

// The solve on the fixed scratch at `base`; *st receives the device status word.
cudaError_t noalloc_solve(unsigned char* base, int n, int nrhs, const double* d_a, int lda, const int* d_ipiv,
                          double* d_b, int ldb, cudaStream_t s, int* st) {
  int* status = reinterpret_cast<int*>(base);
  unsigned char* trsv = base + 256;
  int* perm = reinterpret_cast<int*>(base + 256 + round256(TrsvScratch::bytes(n)));
  cudaError_t e;
  if ((e = cudaMemsetAsync(status, 0, sizeof(int), s)) != cudaSuccess) return e;
  if ((e = lu_perm_from_ipiv(d_ipiv, n, perm, s)) != cudaSuccess) return e;
  if ((e = getrs64(d_a, lda, n, perm, d_b, ldb, nrhs, trsv, status, s)) != cudaSuccess) return e;
  if ((e = check_finite(d_b, ldb, n, nrhs, status, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(st, status, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}

// The warm-up call (n = 0): looks the array up and runs every kernel of the solve once, on a 1 x 1
// system placed in the array itself (both widths of the triangular solve), so that the module's code
// and the array are resident on this device before the caller's allocator takes the memory.
cudaError_t noalloc_warm_up(unsigned char* base, cudaStream_t s, int* st) {
  const size_t off = 1u << 20;  // beyond what an order-1 solve uses of the array
  double* a = reinterpret_cast<double*>(base + off);
  int* ipiv = reinterpret_cast<int*>(base + off + 256);
  double* b = reinterpret_cast<double*>(base + off + 512);
  const double one = 1.0;
  const int piv = 1;
  double rhs[kMaxRhs];
  for (double& v : rhs) v = 1.0;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(a, &one, sizeof one, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(ipiv, &piv, sizeof piv, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(b, rhs, sizeof rhs, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  for (int nrhs : {1, kMaxRhs}) {
    if ((e = noalloc_solve(base, 1, nrhs, a, 1, ipiv, b, 1, s, st)) != cudaSuccess) return e;
    if (*st != kOk) return cudaSuccess;
  }
  return cudaSuccess;
}

}  // namespace
}  // namespace bgpu

extern "C" int bgpu_dgetrs_noalloc(int n, int nrhs, const double* d_a, int lda, const int* d_ipiv, double* d_b,
                                   int ldb, void* stream) {
  using namespace bgpu;
  char msg[256];
  if (n < 0 || nrhs < 1 || nrhs > kMaxRhs || lda < std::max(1, n) || ldb < std::max(1, n)) {
    std::snprintf(msg, sizeof msg, "error: bgpu_dgetrs_noalloc: bad arguments (n %d, nrhs %d in 1..%d, lda %d, ldb %d)",
                  n, nrhs, kMaxRhs, lda, ldb);
    log_message(msg);
    return 1;
  }
  const int nmax = noalloc_max_n();
  if (n > nmax) {
    std::snprintf(msg, sizeof msg,
                  "error: bgpu_dgetrs_noalloc: order %d exceeds %d, the most its fixed %zu MiB device scratch holds", n,
                  nmax, kNoAllocBytes >> 20);
    log_message(msg);
    return 1;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  int st = kOk;
  cudaError_t e = noalloc_base(&base, s);
  if (e == cudaSuccess)
    e = (n == 0) ? noalloc_warm_up(base, s, &st) : noalloc_solve(base, n, nrhs, d_a, lda, d_ipiv, d_b, ldb, s, &st);
  if (e == cudaSuccess) {
    if (st == kOk) return 0;
    std::snprintf(msg, sizeof msg, "error: bgpu_dgetrs_noalloc: %s",
                  st == kWaitTimeout ? "a device-side wait ran out (kernel gave up, no result)"
                                     : "the solution is not finite (NaN or Inf)");
    log_message(msg);
    return 1;
  }
  std::snprintf(msg, sizeof msg, "error: bgpu_dgetrs_noalloc: CUDA error: %s", cudaGetErrorString(e));
  log_message(msg);
  return 1;
}
