// C(m x n, FP32) -= A(m x k) B(k x n) on the B200's 5th-generation tensor cores, BF16 operands with
// FP32 accumulation: the trailing update and triangular-solve updates of the mixed-precision LU
// (mixed.cu).  No counterpart in the reference, whose LU is LAPACK's dgetrf in FP64.
//
// Persistent kernel: one CTA per SM (320 threads, 197 KB of shared memory) walks the 128 x 256
// output tiles blockIdx.x, blockIdx.x + gridDim.x, ... with
//   warp 0, one thread   TMA producer: 128 x 64 tile of A and 256 x 64 tile of B per stage
//                        (cp.async.bulk.tensor, 128-byte swizzle) into a 4-stage ring guarded by
//                        full/empty mbarriers; the ring runs on across tiles
//   warp 1               allocates all 512 TMEM columns (two 256-column FP32 accumulators); one
//                        thread issues tcgen05.mma kind::f16 (M 128, N 256, K 16; A and B K-major in
//                        shared memory), returns each stage with tcgen05.commit and hands a finished
//                        accumulator to the epilogue with another commit
//   warps 2-9            epilogue: tcgen05.ld of an accumulator (warp w reads TMEM lanes
//                        32 (w % 4) .. +31 = tile rows, half of the 256 columns), C -= D in FP32 with
//                        the next 32 columns of C already loaded; then the accumulator is released
// so the epilogue of one tile runs under the main loop of the next.  Operands are BF16 copies in
// K-major layout (A row-major, B column-major), made by the cast kernels below.  Tiles are ordered
// in groups of 16 row-tiles so that the CTAs resident together share A and B slices in L2.  Every
// mbarrier wait is bounded: on expiry the thread records a status and stops issuing work; all roles
// still reach the teardown, which frees TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bgpu_internal.h"

namespace bgpu {
namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr uint32_t kStageA = BM * BK * 2;  // 16 KB
constexpr uint32_t kStageB = BN * BK * 2;  // 32 KB
constexpr uint32_t kSmem = STAGES * (kStageA + kStageB) + 1024 + 256;
// the small-K variant (at most 8 K tiles): two stages and the C tile staged in shared memory (128 x 256
// FP32, four 32 x 256 boxes of 32 KB) for TMA loads and stores
constexpr int kStagesSmallK = 2, kSmallKTiles = 8;
constexpr uint32_t kCBox = 32 * BN * 4;
constexpr uint32_t kSmemStaged = kStagesSmallK * (kStageA + kStageB) + 4 * kCBox + 1024 + 256;
constexpr uint32_t kTmemCols = 512;        // two accumulators of BN columns
constexpr int kGroupM = 16;
constexpr unsigned long long kWaitNs = 2000000000ull;  // a wait gives up after 2 s

// instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
  return t;
}
// Bounded wait; false (status recorded) when it runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    for (int i = 0; i < 256; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kWaitNs) break;
  }
  atomicExch(status, (int)kWaitTimeout);
  return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)tm), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// TMA store of a box from shared memory (bulk-group completion), its commit and waits
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* tm, const void* src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"((uint64_t)tm),
               "r"(x), "r"(y), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, %0;\n" ::"r"(32 * kEpiWarps) : "memory"); }
// Shared-memory matrix descriptor: K-major, 128-byte swizzle; rows of 128 B, 8-row groups 1024 B
// apart (stride byte offset), version 1 (bits 46-47), layout 2 = SWIZZLE_128B (bits 61-63).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}
// D (TMEM) (+)= A B; no output lane disabled.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%"
      "21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// tile index -> (row tile, column tile) in the grouped order
__device__ __forceinline__ void tile_coords(int tile, int tiles_m, int tiles_n, int& tm, int& tn) {
  const int per_group = kGroupM * tiles_n;
  const int group = tile / per_group;
  const int first_m = group * kGroupM;
  const int group_m = min(tiles_m - first_m, kGroupM);
  tm = first_m + (tile % per_group) % group_m;
  tn = (tile % per_group) / group_m;
}

// A's tiles start at row a_y0, column (K) a_x0 of its tensor map; B's at row b_y0, column b_x0 of its
// (both 0 for operand buffers that hold just this product).  stamp (optional): the launch's first
// CTA start and last CTA end on the global nanosecond timer, as atomic min into stamp[0] and max into
// stamp[1] (live per-launch timing that also works inside a CUDA graph).
// NST pipeline stages; STAGED: whole C tiles loaded and stored by TMA through shared memory (tmC the
// C matrix's FP32 map, 32 x 256 boxes; C's element (0, 0) at (c_r0, c_c0) of it), ragged ones by
// plain loads and stores.
template <int NST, bool STAGED>
__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_bf16_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const __grid_constant__ CUtensorMap tmC, int m, int n, int k, float* __restrict__ C, long ldc,
                   int c_r0, int c_c0, int tiles_m, int tiles_n, int* status, int a_y0, int a_x0, int b_y0, int b_x0,
                   unsigned long long* stamp) {
  constexpr int STAGES = NST;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = smem;
  uint8_t* sB = smem + STAGES * kStageA;
  uint8_t* sC = sB + STAGES * kStageB;  // (staged) the C tile: four 32 x 256 boxes
  uint64_t* full = reinterpret_cast<uint64_t*>(sC + (STAGED ? 4 * kCBox : 0));
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;   // [2]
  uint64_t* acc_empty = acc_full + 2;    // [2]
  uint64_t* c_full = acc_empty + 2;      // (staged) the C tile landed
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(c_full + 1);
  int* s_flags = reinterpret_cast<int*>(tmem_slot + 1);  // [0] abort, [1] the epilogue goes on
  volatile int& s_abort = s_flags[0];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = tiles_m * tiles_n;
  const int ktiles = (k + BK - 1) / BK;

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpiWarps);
    }
    mbar_init(c_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // the set-up above overlaps the previous launch's tail under programmatic dependent launch; the
  // operands and C are read only after it has completed
  pdl_wait();
  pdl_trigger();
  if (stamp && threadIdx.x == 0) atomicMin(stamp, global_ns());

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      for (int tile = blockIdx.x; tile < ntiles && !*(volatile int*)&s_abort; tile += gridDim.x) {
        int tm, tn;
        tile_coords(tile, tiles_m, tiles_n, tm, tn);
        for (int kt = 0; kt < ktiles; ++kt, ++it) {
          const uint32_t s = it % STAGES;
          if (it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) & 1) ^ 1, status)) {
            s_abort = 1;
            break;
          }
          if (*(volatile int*)&s_abort) break;
          mbar_expect_tx(&full[s], kStageA + kStageB);
          tma_load_2d(sA + s * kStageA, &tmA, a_x0 + kt * BK, a_y0 + tm * BM, &full[s]);
          tma_load_2d(sB + s * kStageB, &tmB, b_x0 + kt * BK, b_y0 + tn * BN, &full[s]);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0, local = 0;
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++local) {
        const uint32_t b = local & 1, use = local >> 1;
        if (use >= 1 && !mbar_wait(&acc_empty[b], (use - 1) & 1, status)) {
          s_abort = 1;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + b * BN;
        bool ok = true;
        for (int kt = 0; kt < ktiles; ++kt, ++it) {
          const uint32_t s = it % STAGES;
          if (!mbar_wait(&full[s], (it / STAGES) & 1, status)) {
            s_abort = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + s * kStageA), b0 = smem_u32(sB + s * kStageB);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk)
            mma_bf16(acc, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32), (kt > 0 || kk > 0) ? 1u : 0u);
          mma_commit(&empty[s]);
        }
        if (!ok) break;
        mma_commit(&acc_full[b]);
      }
    }
  } else {
    if constexpr (STAGED) {
      // epilogue warp: TMEM lanes 32 q .. 32 q + 31 (tile rows), columns [half * 128, half * 128 + 128);
      // thread et == 0 leads: the TMA traffic of whole tiles and the waits whose outcome all share
      const int q = warp & 3, half = (warp - 2) >> 2, et = threadIdx.x - 64;
      uint32_t local = 0, cuse = 0;
      bool stored = false;  // (leader) a TMA store from sC in flight
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++local) {
        const uint32_t b = local & 1, use = local >> 1;
        int tm, tn;
        tile_coords(tile, tiles_m, tiles_n, tm, tn);
        const bool whole = (tm + 1) * BM <= m && (tn + 1) * BN <= n;
        const int crow0 = c_r0 + tm * BM, ccol0 = c_c0 + tn * BN;
        if (et == 0) {
          bool ok = true;
          if (whole) {
            if (stored) bulk_wait_read();  // the last tile's stores have read sC
            mbar_expect_tx(c_full, 4 * kCBox);
            for (int c = 0; c < 4; ++c) tma_load_2d(sC + c * kCBox, &tmC, crow0 + 32 * c, ccol0, c_full);
          }
          ok = mbar_wait(&acc_full[b], use & 1, status);
          if (ok && whole) ok = mbar_wait(c_full, cuse & 1, status);
          s_flags[1] = ok && !s_abort;
        }
        epi_bar();
        if (!s_flags[1]) {
          if (et == 0) s_abort = 1;
          break;
        }
        tc_fence_after();
        if (whole) {
          mbar_wait(c_full, (cuse++) & 1, status);  // (complete: the leader saw it)
          // sC box q: rows 32 q ..; column j at 128 j bytes, 16-byte group (row & 31) / 4 swizzled with
          // j & 7 (the TMA's 128-byte swizzle)
          uint8_t* cb = sC + q * kCBox + (lane & 3) * 4;
#pragma unroll 1
          for (int c = 0; c < BN / 2 / 32; ++c) {
            float v[32];
            const int j0 = half * (BN / 2) + c * 32;
            tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + b * BN + (uint32_t)j0, v);
#pragma unroll
            for (int jj = 0; jj < 32; ++jj) {
              const int j = j0 + jj;
              float* o = reinterpret_cast<float*>(cb + j * 128 + (((lane >> 2) ^ (j & 7)) << 4));
              *o = *o - v[jj];
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[b]);
          fence_async_smem();
          epi_bar();
          if (et == 0) {
            for (int c = 0; c < 4; ++c) tma_store_2d(&tmC, sC + c * kCBox, crow0 + 32 * c, ccol0);
            bulk_commit();
            stored = true;
          }
          continue;
        }
        // a ragged tile: plain loads and stores, 32 columns at a time
        const int row = tm * BM + q * 32 + lane;
        const bool rok = row < m;
        float* crow = C + row;
#pragma unroll 1
        for (int c = 0; c < BN / 2 / 32; ++c) {
          float v[32];
          const int c0 = tn * BN + half * (BN / 2) + c * 32;
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + b * BN + (uint32_t)(half * (BN / 2) + c * 32), v);
          if (rok) {
            float cv[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) cv[j] = c0 + j < n ? __ldcs(crow + (size_t)(c0 + j) * ldc) : 0.f;
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (c0 + j < n) __stcs(crow + (size_t)(c0 + j) * ldc, cv[j] - v[j]);
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[b]);
      }
      if (et == 0 && stored) bulk_wait_all();
    } else {
      // epilogue warp: TMEM lanes 32 q .. 32 q + 31 (tile rows), columns [half * 128, half * 128 + 128)
      const int q = warp & 3, half = (warp - 2) >> 2;
      uint32_t local = 0;
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++local) {
        const uint32_t b = local & 1, use = local >> 1;
        int tm, tn;
        tile_coords(tile, tiles_m, tiles_n, tm, tn);
        const int row = tm * BM + q * 32 + lane;
        const int cbase = tn * BN + half * (BN / 2);
        const bool rok = row < m;
        float* crow = C + row;
        // C of the first 32 columns, loaded before the accumulator is ready
        float cv[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) cv[j] = (rok && cbase + j < n) ? __ldcs(crow + (size_t)(cbase + j) * ldc) : 0.f;
        if (!mbar_wait(&acc_full[b], use & 1, status) || *(volatile int*)&s_abort) break;
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < BN / 2 / 32; ++c) {
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + b * BN + (uint32_t)(half * (BN / 2) + c * 32), v);
          float nv[32];
          const int c0 = cbase + c * 32, c1 = c0 + 32;
          if (c + 1 < BN / 2 / 32) {
#pragma unroll
            for (int j = 0; j < 32; ++j) nv[j] = (rok && c1 + j < n) ? __ldcs(crow + (size_t)(c1 + j) * ldc) : 0.f;
          }
          if (rok) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (c0 + j < n) __stcs(crow + (size_t)(c0 + j) * ldc, cv[j] - v[j]);
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) cv[j] = nv[j];
        }
        // every tcgen05.ld of this warp has completed (tmem_ld32 waits): release the accumulator
        tc_fence_before();
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&acc_empty[b])) : "memory");
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
  }
  if (stamp && threadIdx.x == 0) {
    __threadfence();
    atomicMax(stamp + 1, global_ns());
  }
}

// ------------------------------------------------------------------------------------------
// Panel products of the FP32 LU on the tensor cores (tcgen05 kind::tf32, FP32 accumulation), a
// 128 x 128 operand R resident in shared memory against a long panel P streamed in 128-long tiles:
//   left:  X (h x len)  (=|-=)  R (h x 128) P (128 x len)
//   right: X (len x h)  (=|-=)  P (len x 128) R (128 x h)
// The triangular-solve leaves are the assigning form (R the inverse of a diagonal block, X = P in
// place, with the BF16 mirror beside it); the K = 128 updates of the recursion (C -= A B with one
// side at most 128) the subtracting form.  Both MMA operands must be K-major (kind::tf32 takes no
// MN-major operand), so the operands that are MN-major in the column-major factor -- the left
// form's R and the right form's P -- arrive by TMA as four 32 x 32 boxes per 32-deep K chunk and
// four transposer warps rewrite each chunk K-major (128 rows of 128 bytes, 128-byte swizzle) before
// the MMA warp uses it.  Shared memory: R (4 chunks of 16 KB), a raw ring (4 x 16 KB, TMA) and an
// operand ring (4 x 16 KB); two TMEM accumulators of 128 x 128 FP32.
constexpr int kPtStages = 4;
constexpr uint32_t kPtChunk = 128 * 32 * 4;  // 16 KB
// R (64 KB), raw and operand rings, the output tile (64 KB: four 32 x 128 FP32 boxes) and its BF16
// mirror (32 KB: two 64 x 128 boxes), barriers
constexpr uint32_t kPtOutOff = 4 * kPtChunk + kPtStages * kPtChunk;
constexpr uint32_t kPtMirOff = kPtOutOff + 4 * kPtChunk;
constexpr uint32_t kPtBarOff = kPtMirOff + 2 * kPtChunk;
constexpr uint32_t kPtSmem = kPtBarOff + 256 + 1024;
constexpr uint32_t kPtTmemCols = 256;
constexpr int kPtTrWarps = 4;
constexpr int kPtThreads = 64 + 32 * kEpiWarps + 32 * kPtTrWarps;
// instruction descriptor, kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2),
// both K-major, N = 128 (>> 3 at bits 17-22), M = 128 (>> 4 at bits 24-28)
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(128 >> 3) << 17) |
                                ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescTf32), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// One 16 KB chunk from four MN-major boxes (box c: MN rows 32 c .. 32 c + 31; K row k at 128 k bytes,
// 16-byte group g of a row at (g ^ (k & 7)) -- the TMA's 128-byte swizzle) to the K-major layout
// (MN row r at 128 r bytes, K group g at (g ^ (r & 7))).  t: 0 .. 127 (the transposer threads); each
// writes 8 groups of 4 K values, a warp 32 consecutive rows (reads and writes free of bank conflicts).
__device__ __forceinline__ void transpose_chunk(const uint8_t* src, uint8_t* dst, int t) {
  const int lane = t & 31, w = t >> 5;
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int mn = lane + 32 * (it & 3), kg = w + 4 * (it >> 2);
    const uint8_t* sb = src + (mn >> 5) * 4096 + (mn & 3) * 4;
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = 4 * kg + e;
      v[e] = *reinterpret_cast<const float*>(sb + k * 128 + ((((mn & 31) >> 2) ^ (k & 7)) << 4));
    }
    *reinterpret_cast<float4*>(dst + mn * 128 + ((kg ^ (mn & 7)) << 4)) = make_float4(v[0], v[1], v[2], v[3]);
  }
}

// transpose_chunk in place: the four transposer warps read all their values, meet at a named
// barrier (id 2) that also ANDs their `ok` (the outcome of each thread's wait for the boxes), then --
// if all were ok -- write (the written places are a permutation of the read ones).  Returns the AND,
// alike in all 128 threads, so they leave a loop together.
__device__ __forceinline__ bool transpose_chunk_inplace(uint8_t* buf, int t, bool ok) {
  const int lane = t & 31, w = t >> 5;
  float v[8][4];
  if (ok) {
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      const int mn = lane + 32 * (it & 3), kg = w + 4 * (it >> 2);
      const uint8_t* sb = buf + (mn >> 5) * 4096 + (mn & 3) * 4;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k = 4 * kg + e;
        v[it][e] = *reinterpret_cast<const float*>(sb + k * 128 + ((((mn & 31) >> 2) ^ (k & 7)) << 4));
      }
    }
  }
  unsigned all;
  asm volatile(
      "{\n .reg .pred pi, po;\n setp.ne.u32 pi, %1, 0;\n bar.red.and.pred po, 2, %2, pi;\n selp.u32 %0, 1, 0, po;\n}\n"
      : "=r"(all)
      : "r"((unsigned)ok), "r"(32 * kPtTrWarps)
      : "memory");
  if (!all) return false;
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const int mn = lane + 32 * (it & 3), kg = w + 4 * (it >> 2);
    *reinterpret_cast<float4*>(buf + mn * 128 + ((kg ^ (mn & 7)) << 4)) = make_float4(v[it][0], v[it][1], v[it][2], v[it][3]);
  }
  return true;
}

// tmR, tmP: R's and P's tensor maps (K-major sources: 32 x 128 boxes, one per K chunk; MN-major
// sources: 32 x 32 boxes).  R starts at (rx0, ry0) of its map, P at (px0, py0): left, R's box
// (rx0 + 32 c, ry0 + 32 kc) and P's (px0 + 32 kc, py0 + 128 tile); right, R's (rx0 + 32 kc, ry0)
// and P's (px0 + 128 tile + 32 c, py0 + 32 kc).  X: the result block (ldx) at row xr0, column xc0
// of the matrix, h its extent along R.  Whole 128 x 128 tiles of X go out (and, subtracting, come
// in) as TMA boxes of the factor's K-major map tmX (32 rows x 128 columns) through shared memory,
// the mirror's as 64 x 128 boxes of tmM (left: column-major mirror at (row, column); right:
// row-major at (column, row)); ragged tiles by plain loads and stores.
template <bool LEFT, bool SUB>
__global__ void __launch_bounds__(kPtThreads, 1)
    k_panel_tf32(const __grid_constant__ CUtensorMap tmR, const __grid_constant__ CUtensorMap tmP,
                 const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmM, int rx0, int ry0,
                 int px0, int py0, int h, int len, float* __restrict__ X, long ldx, int xr0, int xc0,
                 __nv_bfloat16* __restrict__ mir, long ldm, int* status, unsigned long long* stamp) {
  // row group blockIdx.y of a 256-wide R: its 128 rows (left) or columns (right), and X's with them
  if (blockIdx.y) {
    const int o = 128 * blockIdx.y;
    h -= o;
    if (LEFT) {
      rx0 += o, xr0 += o, X += o;
      if (mir) mir += o;
    } else {
      ry0 += o, xc0 += o, X += (size_t)o * ldx;
      if (mir) mir += o;
    }
  }
  h = min(h, 128);
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* sR = smem;                               // R, K-major: 4 chunks
  uint8_t* sOp = smem + 4 * kPtChunk;  // P's K-major chunks (right: the MN-major boxes land there and
                                       // are transposed in place)
  uint8_t* sOut = smem + kPtOutOff;                 // the output tile (left: R's boxes first)
  uint8_t* sMir = smem + kPtMirOff;                 // its BF16 mirror
  uint64_t* raw_full = reinterpret_cast<uint64_t*>(smem + kPtBarOff);
  uint64_t* op_full = raw_full + kPtStages;
  uint64_t* op_empty = op_full + kPtStages;
  uint64_t* acc_full = op_empty + kPtStages;  // [2]
  uint64_t* acc_empty = acc_full + 2;         // [2]
  uint64_t* r_raw = acc_empty + 2;            // left: R's boxes landed
  uint64_t* r_full = r_raw + 1;               // R ready (K-major)
  uint64_t* c_full = r_full + 1;              // (subtracting) the C tile landed
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(c_full + 1);
  int* s_flags = reinterpret_cast<int*>(tmem_slot + 1);  // [0] abort, [1] the epilogue goes on
  volatile int& s_abort = s_flags[0];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = (len + 127) / 128;
  const int tr_first = 2 + kEpiWarps;  // the transposer warps

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < kPtStages; ++s) {
      mbar_init(&raw_full[s], 1);
      mbar_init(&op_full[s], LEFT ? 1 : kPtTrWarps);
      mbar_init(&op_empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpiWarps);
    }
    mbar_init(r_raw, 1);
    mbar_init(r_full, LEFT ? kPtTrWarps : 1);
    mbar_init(c_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kPtTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  pdl_wait();
  pdl_trigger();
  if (stamp && threadIdx.x == 0) atomicMin(stamp, global_ns());

  if (warp == 0) {
    if (lane == 0) {
      if (LEFT) {
        // R's MN-major boxes into the raw ring (free until the transposers have read them)
        mbar_expect_tx(r_raw, 4 * kPtChunk);
        for (int kc = 0; kc < 4; ++kc)
          for (int c = 0; c < 4; ++c) tma_load_2d(sOut + kc * kPtChunk + c * 4096, &tmR, rx0 + 32 * c, ry0 + 32 * kc, r_raw);
      } else {
        mbar_expect_tx(r_full, 4 * kPtChunk);
        for (int kc = 0; kc < 4; ++kc) tma_load_2d(sR + kc * kPtChunk, &tmR, rx0 + 32 * kc, ry0, r_full);
      }
      uint32_t it = 0;
      for (int tile = blockIdx.x; tile < ntiles && !*(volatile int*)&s_abort; tile += gridDim.x) {
        for (int kc = 0; kc < 4; ++kc, ++it) {
          const uint32_t s = it % kPtStages;
          if (it >= kPtStages && !mbar_wait(&op_empty[s], ((it / kPtStages) & 1) ^ 1, status)) {
            s_abort = 1;
            break;
          }
          if (*(volatile int*)&s_abort) break;
          if (LEFT) {
            mbar_expect_tx(&op_full[s], kPtChunk);
            tma_load_2d(sOp + s * kPtChunk, &tmP, px0 + 32 * kc, py0 + 128 * tile, &op_full[s]);
          } else {
            mbar_expect_tx(&raw_full[s], kPtChunk);
            for (int c = 0; c < 4; ++c)
              tma_load_2d(sOp + s * kPtChunk + c * 4096, &tmP, px0 + 128 * tile + 32 * c, py0 + 32 * kc, &raw_full[s]);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      bool ok = mbar_wait(r_full, 0, status);
      if (!ok) s_abort = 1;
      tc_fence_after();
      uint32_t it = 0, local = 0;
      for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x, ++local) {
        const uint32_t b = local & 1, use = local >> 1;
        if (use >= 1 && !mbar_wait(&acc_empty[b], (use - 1) & 1, status)) {
          s_abort = 1;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + b * 128;
        for (int kc = 0; kc < 4; ++kc, ++it) {
          const uint32_t s = it % kPtStages;
          if (!mbar_wait(&op_full[s], (it / kPtStages) & 1, status)) {
            s_abort = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t r0s = smem_u32(sR + kc * kPtChunk), p0s = smem_u32(sOp + s * kPtChunk);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            // K step of 8: 32 bytes along the 128-byte rows of both operands
            const uint64_t rd = sw128_desc(r0s + kk * 32), pd = sw128_desc(p0s + kk * 32);
            mma_tf32(acc, LEFT ? rd : pd, LEFT ? pd : rd, (kc > 0 || kk > 0) ? 1u : 0u);
          }
          mma_commit(&op_empty[s]);
        }
        if (!ok) break;
        mma_commit(&acc_full[b]);
      }
    }
  } else if (warp >= tr_first) {
    const int t = threadIdx.x - 32 * tr_first;
    if (LEFT) {
      if (mbar_wait(r_raw, 0, status) && !*(volatile int*)&s_abort) {
        for (int kc = 0; kc < 4; ++kc) transpose_chunk(sOut + kc * kPtChunk, sR + kc * kPtChunk, t);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(r_full);
      } else {
        s_abort = 1;
      }
    } else {
      uint32_t it = 0;
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        bool ok = true;
        for (int kc = 0; kc < 4; ++kc, ++it) {
          const uint32_t s = it % kPtStages;
          // (the transposition's barrier makes the four warps agree on the waits' outcome)
          if (!transpose_chunk_inplace(sOp + s * kPtChunk, t,
                                       mbar_wait(&raw_full[s], (it / kPtStages) & 1, status) && !s_abort)) {
            s_abort = 1;
            ok = false;
            break;
          }
          fence_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(&op_full[s]);
        }
        if (!ok) break;
      }
    }
  } else {
    // epilogue warp: TMEM lanes 32 q .. 32 q + 31 (the tile's rows), columns [64 half, 64 half + 64);
    // thread et == 0 leads: the TMA traffic of whole tiles and the waits whose outcome all share
    const int q = warp & 3, half = (warp - 2) >> 2;
    const int et = threadIdx.x - 64;
    const int r = q * 32 + lane;  // accumulator row
    uint32_t local = 0, cuse = 0;
    bool stored = false;  // (leader) a TMA store from sOut / sMir in flight
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++local) {
      const uint32_t b = local & 1, use = local >> 1;
      const bool whole = h == 128 && 128 * (tile + 1) <= len;
      const int trow = xr0 + (LEFT ? 0 : 128 * tile), tcol = xc0 + (LEFT ? 128 * tile : 0);  // the tile in X's matrix
      if (et == 0) {
        bool ok = true;
        if (whole) {
          if (stored) bulk_wait_read();                               // the last stores have read sOut, sMir
          if (LEFT && local == 0) ok = mbar_wait(r_full, 0, status);  // sOut held R's boxes until then
          if (SUB && ok) {
            mbar_expect_tx(c_full, 4 * kPtChunk);
            for (int c = 0; c < 4; ++c) tma_load_2d(sOut + c * kPtChunk, &tmX, trow + 32 * c, tcol, c_full);
          }
        }
        ok = ok && mbar_wait(&acc_full[b], use & 1, status);
        if (ok && SUB && whole) ok = mbar_wait(c_full, cuse & 1, status);
        s_flags[1] = ok && !s_abort;
      }
      epi_bar();
      if (!s_flags[1]) {
        if (et == 0) s_abort = 1;
        break;
      }
      if (SUB && whole) mbar_wait(c_full, (cuse++) & 1, status);  // (complete: the leader saw it)
      tc_fence_after();
      if (whole) {
        // sOut box c: rows 32 c .. 32 c + 31; column j at 128 j bytes, 16-byte group (row & 31) / 4
        // swizzled with j & 7 (the TMA's 128-byte swizzle)
        uint8_t* ob = sOut + q * kPtChunk + (lane & 3) * 4;
#pragma unroll 1
        for (int c = 0; c < 2; ++c) {
          float v[32];
          const int j0 = 64 * half + 32 * c;
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + b * 128 + (uint32_t)j0, v);
#pragma unroll
          for (int jj = 0; jj < 32; ++jj) {
            const int j = j0 + jj;
            float* o = reinterpret_cast<float*>(ob + j * 128 + (((lane >> 2) ^ (j & 7)) << 4));
            const float x = SUB ? *o - v[jj] : v[jj];
            *o = x;
            v[jj] = x;
            if (!SUB && LEFT && mir) {
              // column-major mirror box r / 64: column j at 128 j bytes, group (r & 63) / 8 ^ (j & 7)
              *reinterpret_cast<__nv_bfloat16*>(sMir + (r >> 6) * kPtChunk + j * 128 +
                                               ((((r & 63) >> 3) ^ (j & 7)) << 4) + (r & 7) * 2) = __float2bfloat16_rn(x);
            }
          }
          if (!SUB && !LEFT && mir) {
            // row-major mirror box j0 / 64: row r at 128 r bytes, group (j & 63) / 8 ^ (r & 7)
#pragma unroll
            for (int g = 0; g < 4; ++g) {
              uint4 pk;
              uint32_t* w = reinterpret_cast<uint32_t*>(&pk);
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const __nv_bfloat162 two = __floats2bfloat162_rn(v[8 * g + 2 * e], v[8 * g + 2 * e + 1]);
                w[e] = *reinterpret_cast<const uint32_t*>(&two);
              }
              *reinterpret_cast<uint4*>(sMir + (j0 >> 6) * kPtChunk + r * 128 +
                                        (((((j0 & 63) >> 3) + g) ^ (r & 7)) << 4)) = pk;
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[b]);
        fence_async_smem();
        epi_bar();
        if (et == 0) {
          for (int c = 0; c < 4; ++c) tma_store_2d(&tmX, sOut + c * kPtChunk, trow + 32 * c, tcol);
          if (!SUB && mir) {
            for (int c = 0; c < 2; ++c) {
              if (LEFT)
                tma_store_2d(&tmM, sMir + c * kPtChunk, trow + 64 * c, tcol);  // (row, column)
              else
                tma_store_2d(&tmM, sMir + c * kPtChunk, tcol + 64 * c, trow);  // (column, row)
            }
          }
          bulk_commit();
          stored = true;
        }
        continue;
      }
      // left: X row r (valid below h), columns 128 tile + j; right: X row 128 tile + r (valid below len),
      // columns j (valid below h); j = 64 half + 0 .. 63
      const int xrow = LEFT ? r : 128 * tile + r;
      const bool rok = LEFT ? r < h : xrow < len;
      const int jlim = LEFT ? len - 128 * tile : h;  // columns j below jlim are valid
      float* xp = X + (LEFT ? (size_t)(128 * tile) * ldx : (size_t)0) + xrow;
#pragma unroll 1
      for (int c = 0; c < 2; ++c) {
        float v[32];
        const int j0 = 64 * half + 32 * c;
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + b * 128 + (uint32_t)j0, v);
        if constexpr (SUB) {
          // (a ragged tile: C by plain loads, 32 columns at a time)
          if (rok) {
            float cv[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) cv[j] = j0 + j < jlim ? __ldcs(xp + (size_t)(j0 + j) * ldx) : 0.f;
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (j0 + j < jlim) __stcs(xp + (size_t)(j0 + j) * ldx, cv[j] - v[j]);
          }
          continue;
        }
        if (!rok) continue;
        {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (j0 + j < jlim) xp[(size_t)(j0 + j) * ldx] = v[j];
          if (mir) {
            if (LEFT) {
              // column-major mirror: element (r, 128 tile + j)
              __nv_bfloat16* mp = mir + (size_t)(128 * tile) * ldm + r;
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (j0 + j < jlim) mp[(size_t)(j0 + j) * ldm] = __float2bfloat16_rn(v[j]);
            } else {
              // row-major mirror: row xrow, 32 consecutive columns
              __nv_bfloat16* dst = mir + (size_t)xrow * ldm + j0;
              if (j0 + 32 <= jlim && ((reinterpret_cast<uintptr_t>(dst) & 15) == 0)) {
#pragma unroll
                for (int g = 0; g < 4; ++g) {
                  uint4 pk;
                  uint32_t* w = reinterpret_cast<uint32_t*>(&pk);
#pragma unroll
                  for (int e = 0; e < 4; ++e) {
                    const __nv_bfloat162 two = __floats2bfloat162_rn(v[8 * g + 2 * e], v[8 * g + 2 * e + 1]);
                    w[e] = *reinterpret_cast<const uint32_t*>(&two);
                  }
                  *reinterpret_cast<uint4*>(dst + 8 * g) = pk;
                }
              } else {
#pragma unroll
                for (int j = 0; j < 32; ++j)
                  if (j0 + j < jlim) dst[j] = __float2bfloat16_rn(v[j]);
              }
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
    if (et == 0 && stored) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kPtTmemCols));
  }
  if (stamp && threadIdx.x == 0) {
    __threadfence();
    atomicMax(stamp + 1, global_ns());
  }
}

// ------------------------------------------------------------------------------------------
// A triangular-solve leaf 256 deep on the tensor cores (TF32): the inverse of a 256 x 256 diagonal
// block, T^-1 = [[D1, 0], [F, D2]] (lower) or [[E1, G], [0, E2]] (upper) with F = -D2 L21 D1 and
// G = -E1 U12 E2 (k_combine256), applied to the 256-deep panel in one launch instead of leaf, K = 128
// update, leaf:
//   left:  X (256 x len) := Tinv P      right: X (len x 256) := P Tinv
// Each CTA owns whole 128-long tiles of the panel and forms both 128-halves of each (row groups on
// the left, column groups on the right) in two TMEM accumulators before any of the tile is written:
// the result replaces the panel in place, and the second half reads all 256 of the tile's inputs.
// The work of a tile is 12 steps of a 32-deep K chunk: half 0 over K 0..127 (the zero quarter of
// Tinv skipped), half 1 over K 0..255.  Each step brings a K-major chunk by TMA ("direct": P on the
// left, Tinv on the right) and an MN-major one as four 32 x 32 boxes that the four transposer warps
// rewrite K-major ("trans": Tinv on the left, P on the right), the MMA's A operand always the trans
// slot and B the direct one.  The epilogue stages each whole 128 x 128 half through shared memory
// for TMA stores, with the BF16 mirror; ragged halves and tiles by plain stores.
constexpr int kL2Stages = 4;
constexpr uint32_t kL2Stage = 2 * kPtChunk;  // direct, trans (the MN-major boxes land there and are
                                             // transposed in place)
constexpr uint32_t kL2OutOff = kL2Stages * kL2Stage;
constexpr uint32_t kL2MirOff = kL2OutOff + 4 * kPtChunk;
constexpr uint32_t kL2BarOff = kL2MirOff + 2 * kPtChunk;
constexpr uint32_t kL2Smem = kL2BarOff + 256 + 1024;
constexpr uint32_t kL2TmemCols = 512;  // two tiles in flight x two halves x 128 columns
constexpr int kL2Steps = 12;           // (half, K chunk) steps per tile

__device__ __forceinline__ void l2_step(int st, int& half, int& kc) {
  half = st < 4 ? 0 : 1;
  kc = st < 4 ? st : st - 4;
}

// tmT: Tinv's map (left: MN-major 32 x 32 boxes over the column-major 256 x 256 blocks, inner 256;
// right: K-major 32 x 128 boxes), block at outer coordinate t0 (256 per diagonal block); tmP, tmX, tmM
// as k_panel_tf32's (the factor's K-major map for the left P and for X, the MN-major one for the
// right P; the mirror's).  The panel starts at (px0, py0): left P chunk kc at (px0 + 32 kc,
// py0 + 128 tile); right at (px0 + 128 tile + 32 c, py0 + 32 kc).  X at (xr0, xc0) of the factor;
// h <= 256 rows (left) or columns (right) of it.
template <bool LEFT>
__global__ void __launch_bounds__(kPtThreads, 1)
    k_leaf256_tf32(const __grid_constant__ CUtensorMap tmT, const __grid_constant__ CUtensorMap tmP,
                   const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmM, int t0, int px0,
                   int py0, int h, int len, float* __restrict__ X, long ldx, int xr0, int xc0,
                   __nv_bfloat16* __restrict__ mir, long ldm, int* status, unsigned long long* stamp) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* sOut = smem + kL2OutOff;
  uint8_t* sMir = smem + kL2MirOff;
  uint64_t* dir_full = reinterpret_cast<uint64_t*>(smem + kL2BarOff);
  uint64_t* raw_full = dir_full + kL2Stages;  // the MN-major boxes landed in the trans slot
  uint64_t* tr_full = raw_full + kL2Stages;   // ... and are transposed
  uint64_t* st_empty = tr_full + kL2Stages;   // the MMA has read the stage's direct and trans slots
  uint64_t* acc_full = st_empty + kL2Stages;  // [2]
  uint64_t* acc_empty = acc_full + 2;         // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  int* s_flags = reinterpret_cast<int*>(tmem_slot + 1);  // [0] abort, [1] the epilogue goes on
  volatile int& s_abort = s_flags[0];
  auto dir = [&](uint32_t s) { return smem + s * kL2Stage; };
  auto trs = [&](uint32_t s) { return smem + s * kL2Stage + kPtChunk; };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = (len + 127) / 128;
  const int tr_first = 2 + kEpiWarps;

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < kL2Stages; ++s) {
      mbar_init(&dir_full[s], 1);
      mbar_init(&raw_full[s], 1);
      mbar_init(&tr_full[s], kPtTrWarps);
      mbar_init(&st_empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpiWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kL2TmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  pdl_wait();
  pdl_trigger();
  if (stamp && threadIdx.x == 0) atomicMin(stamp, global_ns());

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      for (int tile = blockIdx.x; tile < ntiles && !s_abort; tile += gridDim.x) {
        for (int st = 0; st < kL2Steps; ++st, ++it) {
          int g, kc;
          l2_step(st, g, kc);
          const uint32_t s = it % kL2Stages, ph = ((it / kL2Stages) & 1) ^ 1;
          if (it >= kL2Stages && !mbar_wait(&st_empty[s], ph, status)) {
            s_abort = 1;
            break;
          }
          if (s_abort) break;
          mbar_expect_tx(&dir_full[s], kPtChunk);
          mbar_expect_tx(&raw_full[s], kPtChunk);
          if (LEFT) {
            tma_load_2d(dir(s), &tmP, px0 + 32 * kc, py0 + 128 * tile, &dir_full[s]);
            for (int c = 0; c < 4; ++c) tma_load_2d(trs(s) + c * 4096, &tmT, 128 * g + 32 * c, t0 + 32 * kc, &raw_full[s]);
          } else {
            tma_load_2d(dir(s), &tmT, 32 * kc, t0 + 128 * g, &dir_full[s]);
            for (int c = 0; c < 4; ++c)
              tma_load_2d(trs(s) + c * 4096, &tmP, px0 + 128 * tile + 32 * c, py0 + 32 * kc, &raw_full[s]);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0, local = 0;
      bool ok = true;
      for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x, ++local) {
        const uint32_t b = local & 1, use = local >> 1;
        if (use >= 1 && !mbar_wait(&acc_empty[b], (use - 1) & 1, status)) {
          s_abort = 1;
          break;
        }
        tc_fence_after();
        for (int st = 0; st < kL2Steps; ++st, ++it) {
          int g, kc;
          l2_step(st, g, kc);
          const uint32_t s = it % kL2Stages, ph = (it / kL2Stages) & 1;
          if (!mbar_wait(&dir_full[s], ph, status) || !mbar_wait(&tr_full[s], ph, status)) {
            s_abort = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t acc = tmem + (b * 2 + g) * 128;
          const uint32_t a0 = smem_u32(trs(s)), b0 = smem_u32(dir(s));
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            mma_tf32(acc, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32), (kc > 0 || kk > 0) ? 1u : 0u);
          mma_commit(&st_empty[s]);
        }
        if (!ok) break;
        mma_commit(&acc_full[b]);
      }
    }
  } else if (warp >= tr_first) {
    const int t = threadIdx.x - 32 * tr_first;
    uint32_t it = 0;
    bool ok = true;
    for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
      for (int st = 0; st < kL2Steps; ++st, ++it) {
        const uint32_t s = it % kL2Stages, ph = (it / kL2Stages) & 1;
        // the in-place transposition's barrier makes the four warps agree on the waits' outcome
        if (!transpose_chunk_inplace(trs(s), t, mbar_wait(&raw_full[s], ph, status) && !s_abort)) {
          s_abort = 1;
          ok = false;
          break;
        }
        fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tr_full[s]);
      }
    }
  } else {
    // epilogue warp: TMEM lanes 32 q .. 32 q + 31 (the tile's rows), columns [64 cw, 64 cw + 64) of each
    // half's accumulator; thread et == 0 leads (the TMA stores and the waits whose outcome all share)
    const int q = warp & 3, cw = (warp - 2) >> 2;
    const int et = threadIdx.x - 64;
    const int r = q * 32 + lane;  // accumulator row
    uint32_t local = 0;
    bool stored = false;  // (leader) a TMA store from sOut / sMir in flight
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++local) {
      const uint32_t b = local & 1, use = local >> 1;
      if (et == 0) s_flags[1] = mbar_wait(&acc_full[b], use & 1, status) && !s_abort;
      epi_bar();
      if (!s_flags[1]) {
        if (et == 0) s_abort = 1;
        break;
      }
      tc_fence_after();
      for (int g = 0; g < 2; ++g) {
        const int hg = min(h - 128 * g, 128);  // rows (left) or columns (right) of X in this half
        if (hg <= 0) break;
        const bool whole = hg == 128 && 128 * (tile + 1) <= len;
        const int trow = xr0 + (LEFT ? 128 * g : 128 * tile), tcol = xc0 + (LEFT ? 128 * tile : 128 * g);
        const uint32_t accb = tmem + ((uint32_t)(q * 32) << 16) + (b * 2 + g) * 128;
        if (whole) {
          if (et == 0 && stored) bulk_wait_read();  // the last stores have read sOut, sMir
          epi_bar();
          // sOut box q: rows 32 q ..; column j at 128 j bytes, 16-byte group (row & 31) / 4 swizzled with
          // j & 7 (the TMA's 128-byte swizzle)
          uint8_t* ob = sOut + q * kPtChunk + (lane & 3) * 4;
#pragma unroll 1
          for (int c = 0; c < 2; ++c) {
            float v[32];
            const int j0 = 64 * cw + 32 * c;
            tmem_ld32(accb + (uint32_t)j0, v);
#pragma unroll
            for (int jj = 0; jj < 32; ++jj) {
              const int j = j0 + jj;
              *reinterpret_cast<float*>(ob + j * 128 + (((lane >> 2) ^ (j & 7)) << 4)) = v[jj];
              if (LEFT && mir)
                *reinterpret_cast<__nv_bfloat16*>(sMir + (r >> 6) * kPtChunk + j * 128 +
                                                 ((((r & 63) >> 3) ^ (j & 7)) << 4) + (r & 7) * 2) =
                    __float2bfloat16_rn(v[jj]);
            }
            if (!LEFT && mir) {
#pragma unroll
              for (int gg = 0; gg < 4; ++gg) {
                uint4 pk;
                uint32_t* w = reinterpret_cast<uint32_t*>(&pk);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                  const __nv_bfloat162 two = __floats2bfloat162_rn(v[8 * gg + 2 * e], v[8 * gg + 2 * e + 1]);
                  w[e] = *reinterpret_cast<const uint32_t*>(&two);
                }
                *reinterpret_cast<uint4*>(sMir + (j0 >> 6) * kPtChunk + r * 128 +
                                          (((((j0 & 63) >> 3) + gg) ^ (r & 7)) << 4)) = pk;
              }
            }
          }
          fence_async_smem();
          epi_bar();
          if (et == 0) {
            for (int c = 0; c < 4; ++c) tma_store_2d(&tmX, sOut + c * kPtChunk, trow + 32 * c, tcol);
            if (mir) {
              for (int c = 0; c < 2; ++c) {
                if (LEFT)
                  tma_store_2d(&tmM, sMir + c * kPtChunk, trow + 64 * c, tcol);  // (row, column)
                else
                  tma_store_2d(&tmM, sMir + c * kPtChunk, tcol + 64 * c, trow);  // (column, row)
              }
            }
            bulk_commit();
            stored = true;
          }
        } else {
          // a ragged half: plain stores.  Left: X (128 g + r, 128 tile + j); right: X (128 tile + r,
          // 128 g + j)
          const int xi = LEFT ? 128 * g + r : 128 * tile + r;
          const bool rok = LEFT ? r < hg : 128 * tile + r < len;
          const int jbase = LEFT ? 128 * tile : 128 * g;
          const int jlim = LEFT ? len - 128 * tile : hg;
#pragma unroll 1
          for (int c = 0; c < 2; ++c) {
            float v[32];
            const int j0 = 64 * cw + 32 * c;
            tmem_ld32(accb + (uint32_t)j0, v);
            if (!rok) continue;
#pragma unroll
            for (int jj = 0; jj < 32; ++jj) {
              const int j = j0 + jj;
              if (j < jlim) {
                X[(size_t)(jbase + j) * ldx + xi] = v[jj];
                if (mir) {
                  if (LEFT)
                    mir[(size_t)(jbase + j) * ldm + xi] = __float2bfloat16_rn(v[jj]);
                  else
                    mir[(size_t)xi * ldm + jbase + j] = __float2bfloat16_rn(v[jj]);
                }
              }
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
    if (et == 0 && stored) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kL2TmemCols));
  }
  if (stamp && threadIdx.x == 0) {
    __threadfence();
    atomicMax(stamp + 1, global_ns());
  }
}

__global__ void k_stamps_reset(unsigned long long* stamps, int slots) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += gridDim.x * blockDim.x) {
    stamps[2 * i] = ~0ull;
    stamps[2 * i + 1] = 0ull;
  }
}

// ------------------------------------------------------------------------------------------
// BF16 operand copies
// ------------------------------------------------------------------------------------------
// At (m x k row-major, lda_t) = bf16(A), A m x k column-major FP32 (lda): transposed through a
// 32 x 32 shared tile so both sides are coalesced.
// Columns [k, kpad) of At are written as zeros (the GEMM reads whole 64-wide K tiles).
__global__ void k_cast_transpose_bf16(const float* __restrict__ A, long lda, int m, int k, int kpad,
                                      __nv_bfloat16* __restrict__ At, long lda_t) {
  __shared__ float t[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int kk = k0 + r, i = i0 + threadIdx.x;
    t[r][threadIdx.x] = (kk < k && i < m) ? A[(size_t)kk * lda + i] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, kk = k0 + threadIdx.x;
    if (i < m && kk < kpad) At[(size_t)i * lda_t + kk] = __float2bfloat16_rn(t[threadIdx.x][r]);
  }
}

// Bt (k x n column-major, ldb_t) = bf16(B), B k x n column-major FP32 (ldb); 32 x 32 tiles; rows
// [k, kpad) of Bt are written as zeros.
__global__ void k_cast_bf16(const float* __restrict__ B, long ldb, int k, int kpad, int n,
                            __nv_bfloat16* __restrict__ Bt, long ldb_t) {
  const int k0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const int kk = k0 + threadIdx.x;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r;
    if (kk < kpad && j < n) Bt[(size_t)j * ldb_t + kk] = __float2bfloat16_rn(kk < k ? B[(size_t)j * ldb + kk] : 0.f);
  }
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

// 2-D BF16 tensor map: `rows` rows of `cols` elements (row pitch ld elements), box 64 x box_rows,
// 128-byte swizzle, zero fill outside.
bool make_map(CUtensorMap* tm, const void* base, int rows, int cols, long ld, int box_rows) {
  EncodeTiled fn = encoder();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2-D FP32 tensor map: `outer` rows of `inner` elements (pitch ld elements), box 32 x box_outer,
// 128-byte swizzle, zero fill outside.
bool make_map_f32(CUtensorMap* tm, const void* base, long inner, long outer, long ld, int box_outer) {
  EncodeTiled fn = encoder();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {32u, (cuuint32_t)box_outer};
  cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// one CTA per SM (at most one per tile)
int persistent_grid(int tiles) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return std::min(tiles, sms);
}

}  // namespace

cudaError_t cast_transpose_bf16(const float* A, long lda, int m, int k, void* At, long lda_t, cudaStream_t s) {
  if (m <= 0 || k <= 0) return cudaSuccess;
  const int kpad = (k + BK - 1) / BK * BK;
  if (kpad > lda_t) return cudaErrorInvalidValue;
  dim3 grid((m + 31) / 32, (kpad + 31) / 32);
  k_cast_transpose_bf16<<<grid, dim3(32, 8), 0, s>>>(A, lda, m, k, kpad, static_cast<__nv_bfloat16*>(At), lda_t);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t cast_bf16(const float* B, long ldb, int k, int n, void* Bt, long ldb_t, cudaStream_t s) {
  if (k <= 0 || n <= 0) return cudaSuccess;
  const int kpad = (k + BK - 1) / BK * BK;
  if (kpad > ldb_t) return cudaErrorInvalidValue;
  dim3 grid((kpad + 31) / 32, (n + 31) / 32);
  k_cast_bf16<<<grid, dim3(32, 8), 0, s>>>(B, ldb, k, kpad, n, static_cast<__nv_bfloat16*>(Bt), ldb_t);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// Tensor maps over whole BF16 operand buffers (rows x ld elements), built once per buffer: a GEMM
// on a leading part of the buffer reads rows beyond m or n (never stored) and K padding (zeroed by
// the casts).
bool tc_operand_maps(const void* At, int rows_a, long lda_t, const void* Bt, int rows_b, long ldb_t, void* map_a,
                     void* map_b) {
  if ((lda_t % 8) || (ldb_t % 8) || ((uintptr_t)At & 15) || ((uintptr_t)Bt & 15)) return false;
  return make_map(static_cast<CUtensorMap*>(map_a), At, rows_a, (int)lda_t, lda_t, BM) &&
         make_map(static_cast<CUtensorMap*>(map_b), Bt, rows_b, (int)ldb_t, ldb_t, BN);
}

cudaError_t tc_gemm_prepare() {
  cudaError_t e =
      cudaFuncSetAttribute(k_gemm_bf16_tc<STAGES, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_gemm_bf16_tc<kStagesSmallK, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSmemStaged);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_leaf256_tf32<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kL2Smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_leaf256_tf32<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kL2Smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_panel_tf32<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPtSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_panel_tf32<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPtSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_panel_tf32<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPtSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_panel_tf32<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPtSmem);
  return e;
}

bool tc_panel_maps(const float* lu32, int n, long ld, const float* dl, const float* du, void* maps) {
  if ((ld % 4) || ((uintptr_t)lu32 & 15) || ((uintptr_t)dl & 15) || ((uintptr_t)du & 15) || n <= 0) return false;
  CUtensorMap* m = static_cast<CUtensorMap*>(maps);
  const long diag_rows = (long)((n + 127) / 128) * 128;
  return make_map_f32(&m[kMapDL], dl, 128, diag_rows, 128, 32) &&    // MN-major boxes
         make_map_f32(&m[kMapDU], du, 128, diag_rows, 128, 128) &&   // K-major boxes
         make_map_f32(&m[kMapK], lu32, n, n, ld, 128) &&             // K-major boxes
         make_map_f32(&m[kMapMN], lu32, n, n, ld, 32) &&             // MN-major boxes
         make_map_f32(&m[kMapC], lu32, n, n, ld, 256);               // the BF16 GEMM's C tiles
}

bool tc_mirror_store_maps(const void* Am, const void* Bm, int n, long ldm, void* maps) {
  if ((ldm % 8) || ((uintptr_t)Am & 15) || ((uintptr_t)Bm & 15) || n <= 0) return false;
  CUtensorMap* m = static_cast<CUtensorMap*>(maps);
  return make_map(&m[0], Bm, n, n, ldm, 128) &&  // left leaves: column-major mirror, boxes 64 rows x 128
         make_map(&m[1], Am, n, n, ldm, 128);    // right leaves: row-major mirror, boxes 64 columns x 128
}

bool tc_leaf256_maps(const float* dl256, const float* du256, int slots, void* maps) {
  if (((uintptr_t)dl256 & 15) || ((uintptr_t)du256 & 15) || slots <= 0) return false;
  CUtensorMap* m = static_cast<CUtensorMap*>(maps);
  return make_map_f32(&m[0], dl256, 256, (long)slots * 256, 256, 32) &&  // left: MN-major boxes
         make_map_f32(&m[1], du256, 256, (long)slots * 256, 256, 128);   // right: K-major boxes
}

cudaError_t leaf256_tf32(bool left, const void* maps, const void* t_maps, const void* mirror_maps, int slot, int kd,
                         int p0, int h, int len, float* X, long ldx, void* mir, long ldm, int* d_status, cudaStream_t s,
                         unsigned long long* stamp) {
  if (len <= 0 || h <= 0) return cudaSuccess;
  const int xr0 = left ? kd : p0, xc0 = left ? p0 : kd;
  if (h > 256 || (kd % 8) || (p0 % 8) || slot < 0 || (mir && !mirror_maps)) return cudaErrorInvalidValue;
  const CUtensorMap* m = static_cast<const CUtensorMap*>(maps);
  const CUtensorMap* tm = static_cast<const CUtensorMap*>(t_maps) + (left ? 0 : 1);
  const CUtensorMap* mm = mir ? static_cast<const CUtensorMap*>(mirror_maps) + (left ? 0 : 1) : &m[kMapK];
  const dim3 grid(persistent_grid((len + 127) / 128)), block(kPtThreads);
  __nv_bfloat16* mb = static_cast<__nv_bfloat16*>(mir);
  // left P: the K-major map, panel rows kd.., columns p0..; right P: the MN-major map, rows p0..,
  // columns kd..
  const cudaError_t e =
      left ? launch_dependent(k_leaf256_tf32<true>, grid, block, kL2Smem, s, *tm, m[kMapK], m[kMapK], *mm, 256 * slot,
                              kd, p0, h, len, X, ldx, xr0, xc0, mb, ldm, d_status, stamp)
           : launch_dependent(k_leaf256_tf32<false>, grid, block, kL2Smem, s, *tm, m[kMapMN], m[kMapK], *mm,
                              256 * slot, p0, kd, h, len, X, ldx, xr0, xc0, mb, ldm, d_status, stamp);
  BGPU_COUNT_LAUNCH();
  return e;
}

cudaError_t panel_tf32(bool left, bool sub, const void* maps, int map_r, int map_p, const void* mirror_maps, int rx0,
                       int ry0, int px0, int py0, int h, int len, float* X, long ldx, int xr0, int xc0, void* mir,
                       long ldm, int* d_status, cudaStream_t s, unsigned long long* stamp) {
  if (len <= 0 || h <= 0) return cudaSuccess;
  // TMA: the innermost coordinate of every box a multiple of 16 bytes (4 FP32, 8 BF16 elements)
  if (h > 256 || (rx0 % 4) || (px0 % 4) || (xr0 % 4) || map_r < 0 || map_p < 0 || map_r > 3 || map_p > 3 ||
      xr0 < 0 || xc0 < 0 || (h > 128 && !sub))
    return cudaErrorInvalidValue;
  if (mir && (!mirror_maps || (left ? xr0 % 8 : xc0 % 8))) return cudaErrorInvalidValue;
  const CUtensorMap* m = static_cast<const CUtensorMap*>(maps);
  const CUtensorMap* mm = mir ? static_cast<const CUtensorMap*>(mirror_maps) + (left ? 0 : 1) : &m[kMapK];
  const dim3 grid(persistent_grid((len + 127) / 128), (h + 127) / 128), block(kPtThreads);
  __nv_bfloat16* mb = static_cast<__nv_bfloat16*>(mir);
  auto kern = left ? (sub ? k_panel_tf32<true, true> : k_panel_tf32<true, false>)
                   : (sub ? k_panel_tf32<false, true> : k_panel_tf32<false, false>);
  const cudaError_t e = launch_dependent(kern, grid, block, kPtSmem, s, m[map_r], m[map_p], m[kMapK], *mm, rx0, ry0, px0,
                                         py0, h, len, X, ldx, xr0, xc0, mb, ldm, d_status, stamp);
  BGPU_COUNT_LAUNCH();
  return e;
}

// (tc_gemm_prepare must have run: the launch may be captured into a graph)
cudaError_t gemm_bf16_tc_minus_maps(int m, int n, int k, const void* map_a, const void* map_b, float* C, long ldc,
                                    int* d_status, cudaStream_t s, unsigned long long* stamp) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  const CUtensorMap& ma = *static_cast<const CUtensorMap*>(map_a);
  const cudaError_t e = launch_dependent(k_gemm_bf16_tc<STAGES, false>, dim3(persistent_grid(tiles_m * tiles_n)),
                                         dim3(kThreads), kSmem, s, ma, *static_cast<const CUtensorMap*>(map_b), ma, m,
                                         n, k, C, ldc, 0, 0, tiles_m, tiles_n, d_status, 0, 0, 0, 0, stamp);
  BGPU_COUNT_LAUNCH();
  return e;
}

cudaError_t stamps_reset(unsigned long long* stamps, int slots, cudaStream_t s) {
  if (slots <= 0) return cudaSuccess;
  k_stamps_reset<<<(slots + 255) / 256, 256, 0, s>>>(stamps, slots);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

// Tensor maps over two n x n BF16 mirrors of a matrix (Am row-major, Bm column-major, leading
// dimension ldm elements): a product then names its operands by position, with no copies.
bool tc_mirror_maps(const void* Am, const void* Bm, int n, long ldm, void* map_a, void* map_b) {
  if ((ldm % 8) || ((uintptr_t)Am & 15) || ((uintptr_t)Bm & 15)) return false;
  return make_map(static_cast<CUtensorMap*>(map_a), Am, n, n, ldm, BM) &&
         make_map(static_cast<CUtensorMap*>(map_b), Bm, n, n, ldm, BN);
}

// C (m x n) -= A B with A at (a_row, a_k) of map_a's matrix and B at (b_row = first column of B,
// b_k = first row of B) of map_b's (column-major) matrix; a_k and b_k multiples of 8, k a multiple
// of 64.
cudaError_t gemm_bf16_tc_minus_at(int m, int n, int k, const void* map_a, int a_row, int a_k, const void* map_b,
                                  int b_row, int b_k, float* C, long ldc, int* d_status, cudaStream_t s,
                                  unsigned long long* stamp, const void* map_c, int c_row, int c_col) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  if ((a_k % 8) || (b_k % 8) || (k % BK) || (map_c && ((c_row % 4) || c_row < 0 || c_col < 0)))
    return cudaErrorInvalidValue;
  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  const CUtensorMap& ma = *static_cast<const CUtensorMap*>(map_a);
  const CUtensorMap& mb = *static_cast<const CUtensorMap*>(map_b);
  const dim3 grid(persistent_grid(tiles_m * tiles_n));
  cudaError_t e;
  if (map_c && k / BK <= kSmallKTiles)
    e = launch_dependent(k_gemm_bf16_tc<kStagesSmallK, true>, grid, dim3(kThreads), kSmemStaged, s, ma, mb,
                         *static_cast<const CUtensorMap*>(map_c), m, n, k, C, ldc, c_row, c_col, tiles_m, tiles_n,
                         d_status, a_row, a_k, b_row, b_k, stamp);
  else
    e = launch_dependent(k_gemm_bf16_tc<STAGES, false>, grid, dim3(kThreads), kSmem, s, ma, mb, ma, m, n, k, C, ldc, 0,
                         0, tiles_m, tiles_n, d_status, a_row, a_k, b_row, b_k, stamp);
  BGPU_COUNT_LAUNCH();
  return e;
}

// C (m x n FP32, ldc) -= At^T-major A (m x k, row-major BF16, lda_t) * B (k x n column-major BF16,
// ldb_t).  lda_t and ldb_t: multiples of 8 elements; At and Bt 16-byte aligned.
cudaError_t gemm_bf16_tc_minus(int m, int n, int k, const void* At, long lda_t, const void* Bt, long ldb_t, float* C,
                               long ldc, int* d_status, cudaStream_t s) {
  if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
  if ((lda_t % 8) || (ldb_t % 8) || ((uintptr_t)At & 15) || ((uintptr_t)Bt & 15)) return cudaErrorInvalidValue;
  CUtensorMap ta, tb;
  if (!make_map(&ta, At, m, k, lda_t, BM) || !make_map(&tb, Bt, n, k, ldb_t, BN)) return cudaErrorInvalidValue;
  static bool attr = false;
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(k_gemm_bf16_tc<STAGES, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  k_gemm_bf16_tc<STAGES, false><<<persistent_grid(tiles_m * tiles_n), kThreads, kSmem, s>>>(
      ta, tb, ta, m, n, k, C, ldc, 0, 0, tiles_m, tiles_n, d_status, 0, 0, 0, 0, nullptr);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace bgpu
