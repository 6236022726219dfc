// Internal declarations shared by the CUDA translation units and the C-ABI layer of libbestgpu.
// Nothing here is part of the public interface (include/best_hmatrix.h, include/best_gpu.h).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace bgpu {

// Kernel launches issued by the library since it was loaded (bgpu_launch_count).
extern unsigned long long g_launches;
#define BGPU_COUNT_LAUNCH() (++::bgpu::g_launches)

// Device status codes written by kernels into a status word (0 = ok).  Kernels never trap: a
// bounded wait that runs out, or an index check that fails, records a code here and returns.
enum DevStatus : int {
  kOk = 0,
  kWaitTimeout = 1,   // a grid barrier or a dependency flag was not reached in time
  kBadIndex = 2,      // an index check failed (the access was skipped)
  kNotFinite = 3,     // a result is NaN or Inf
};

// Programmatic dependent launch (the factorisation's chain of small launches): a kernel launched
// by launch_dependent may start while the previous kernel of its stream finishes; it calls
// pdl_wait() before it touches anything that kernel writes (every kernel so launched does so first),
// then pdl_trigger() so that the next launch of the stream can start in turn.  Launched the ordinary
// way, both are no-ops.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                   Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#endif

// Per-triangle source geometry on the device: p1, p2, p3 (9 doubles), corrected area, 2 pad.
constexpr int kGeoStride = 12;
// Incenter: x, y, z, pad.
constexpr int kXcStride = 4;

struct DevMesh {
  int n = 0;
  double cg = 1.0;
  double afac = 1.0;
  const double* geo = nullptr;  // n * kGeoStride
  double* xc = nullptr;         // n * kXcStride (written by the self-block kernel)
  double* self9 = nullptr;      // n * 9, self block of triangle t: self9[9t + 3a + b]
  // the mesh's extent lies in [1e-20, 1e20] (mesh_fast_ok): the mixed path's assembly may form one
  // reciprocal of three denominators' product (10th power of the size); otherwise it runs the exact
  // kernel
  bool fast_ok = true;
};
// true when the bounding box of the points (count coordinates, point p's axis a at
// p[a * stride_axis + p * stride_point]) has its largest side in [1e-20, 1e20]
bool mesh_fast_ok(const double* v, long count, long stride_point, long stride_axis);

// The normal-field deflation applied in the assembly epilogue (best/best.f:406-425):
// GR(I,J) += (gdef[comp[J/3]-1] * xmu[J]) * xmu[I] when comp[I/3] == comp[J/3].
struct DevDeflation {
  int ndef = 0;  // 0: none
  const double* gdef = nullptr;
  const int* comp = nullptr;  // 1-based surface of each triangle (nullptr when ndef == 1)
  const double* xmu = nullptr;
};

// Opt-in live timing of one kernel's launches: CUDA events recorded around each launch on its
// stream, summed on read (bgpu_kernel_stats).  Ids as in best_gpu.h (BGPU_KERNEL_*).
struct KernelTimer {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  size_t used = 0;
  double work = 0;
  void begin(cudaStream_t s);
  void end(cudaStream_t s, double w);
  void enable(bool v);
  // launches recorded, their summed device time (ms) and work, then reset (synchronises)
  void read(int* launches, double* ms, double* w);
  // launches timed by other means (device stamps inside a graph), added to the next read
  int extra_launches = 0;
  double extra_ms = 0;
  void add(int launches, double ms, double w) {
    if (!on) return;
    extra_launches += launches;
    extra_ms += ms;
    work += w;
  }
};
constexpr int kTimedKernels = 2;
KernelTimer& kernel_timer(int id);

// driver.cpp: d(D_t, D_r)/d(raw friction blocks Ktt, Ktr, Krt, Krr), each row-major [j][i].
void difco_post_gradient(const double K[4][9], double cg, double dDt[4][9], double dDr[4][9]);

// Queues a message for bhm_log_line (api.cpp).
void log_message(const char* msg);

// assemble.cu -------------------------------------------------------------------------------
cudaError_t launch_self_blocks(const DevMesh& m, cudaStream_t s);
// GR rows of targets [r0,r1) x columns of sources [c0,c1) into out (column-major, ld), entry
// (3(n1-r0)+a, 3(n2-c0)+b).  With defl.ndef > 0 the deflation term is added; with out32 != nullptr
// a single-precision copy (rounded to nearest) is written too (leading dimension ld32).
cudaError_t launch_assemble(const DevMesh& m, int r0, int r1, int c0, int c1, double* out, long ld,
                            const DevDeflation& defl, float* out32, long ld32, cudaStream_t s);
// The same matrix for the mixed path with fewer FP64 operations (assemble_fast.cu): entries within a
// few ulp of launch_assemble's, not bit-compatible with the reference.
cudaError_t launch_assemble_fast(const DevMesh& m, int r0, int r1, int c0, int c1, double* out, long ld,
                                 const DevDeflation& defl, float* out32, long ld32, cudaStream_t s);
// Every mesh of a series at once (whole GR of each, with its deflation): mesh i into out[i] (ld[i]).
constexpr int kMaxSeries = 16;
struct SeriesAssembly {
  int count = 0;
  DevMesh mesh[kMaxSeries];
  DevDeflation defl[kMaxSeries];
  double* out[kMaxSeries] = {};
  long ld[kMaxSeries] = {};
  int tile0[kMaxSeries] = {};  // (filled by the launcher)
};
cudaError_t launch_assemble_series(const SeriesAssembly& sa, cudaStream_t s);
// BEST's mean of GR's diagonal (best/best.f:401-403), summed in BEST's order, into *d_out.
cudaError_t launch_diag_mean(const DevMesh& m, double* d_out, cudaStream_t s);

// BEST's input set-up on the device (geometry.cu): from the triangles as read (n x 9, device), the
// centred mesh in the solver's layout and as BEST's V1, V2, V3 (v: 9 n doubles, v1 | v2 | v3, each n x 3
// column-major), the corrected areas, scal = {AFAC, total area, centroid x, y, z}, COMPON's
// 1-based surfaces and counts = {surfaces, open edges, NDEF}.
struct SetupOut {
  double* geo = nullptr;
  double* v = nullptr;
  double* area = nullptr;
  double* scal = nullptr;
  int* icomp = nullptr;
  int* counts = nullptr;
};
size_t setup_scratch_bytes(int n);
cudaError_t setup_device(int n, const double* tri, int iarea, double truearea, const SetupOut& o, void* scratch,
                         int* status, cudaStream_t s);
// XMU (3 n) and GDEF (ndef) from the mesh, the surfaces and the device's DIAGM (*diagm).
cudaError_t deflation_device(int n, int ndef, const double* geo, const int* icomp, const double* diagm, double* xmu,
                             double* gdef, cudaStream_t s);

// lu.cu -------------------------------------------------------------------------------------
// Scratch for the factorisation kernels (grid barrier words, pivot candidates, status).
struct LuScratch {
  void* base = nullptr;
  size_t bytes = 0;
};
size_t lu_scratch_bytes(int n);
// dgetrf semantics: A (n x n, column-major, lda) overwritten by L and U, ipiv 1-based row
// interchanges, *d_info = 0 or the first exactly-zero pivot (1-based).  d_status receives a
// DevStatus.  Host-side errors return a cudaError_t.
cudaError_t lu64_getrf(double* A, long lda, int n, int* ipiv, int* d_info, int* d_status, const LuScratch& ws,
                       cudaStream_t s);
// The same on up to 16 independent matrices at once: each step's leaves, interchanges, triangular
// solves and updates of all matrices run as one launch each (the matrices' results are those of
// factoring each alone).
struct LuItem {
  double* A;
  long lda;
  int n;
  int* ipiv;  // device, n entries
  int* info;  // device, one int
};
cudaError_t lu64_getrf_batch(const LuItem* items, int count, int* d_status, const LuScratch& ws, cudaStream_t s);
// DGEMM tile-shape autotuner: on = tune the shapes of new GEMM sizes as they are met (outside stream
// capture); the table of choices as text.
void lu_autotune(bool on);
std::string lu_autotune_table();
// kernel attributes of the LU, once, before any stream capture
cudaError_t lu_prepare();
// C(m x n) -= A(m x k) B(k x n), all column-major (FP64 tensor-core path).
cudaError_t dgemm_nn_minus(int m, int n, int k, const double* A, long lda, const double* B, long ldb, double* C,
                           long ldc, cudaStream_t s);

// solve.cu ----------------------------------------------------------------------------------
// The row permutation of a factorisation: perm[i] = original row of row i of P A (0-based).
cudaError_t lu_perm_from_ipiv(const int* ipiv, int n, int* perm, cudaStream_t s);
size_t trsv_scratch_bytes(int n);
// X (n x nrhs, ldx) := A^{-1} X given the LU factors and perm, dgetrs('N') semantics.
cudaError_t getrs64(const double* LU, long lda, int n, const int* perm, double* X, long ldx, int nrhs, void* scratch,
                    int* d_status, cudaStream_t s);
// Inverses of the 128 x 128 diagonal blocks of LU factors (DL: unit-lower parts, DU: upper parts),
// each diag_inverse_elems(n) elements; and the solves that use them.
size_t diag_inverse_elems(int n);
cudaError_t diag_inverses64(const double* LU, long lda, int n, double* DL, double* DU, cudaStream_t s);
cudaError_t getrs64_inv(const double* LU, long lda, const double* DL, const double* DU, int n, const int* perm,
                        double* X, long ldx, int nrhs, void* scratch, int* d_status, cudaStream_t s);
// dgetrs('T'): X := A^-T X with the same factors (the adjoint solve).
cudaError_t getrs64_trans_inv(const double* LU, long lda, const double* DL, const double* DU, int n, const int* perm,
                              double* X, long ldx, int nrhs, void* scratch, int* d_status, cudaStream_t s);
// Y := U^-1 L^-1 Y, FP32 factors, right-hand sides and sums (the mixed path's preconditioner)
cudaError_t trsv_lu32_inv(const float* LU, long lda, const float* DL, const float* DU, const float* WL,
                          const float* WU, int n, float* Y, long ldy, int nrhs, void* scratch, int* d_status,
                          cudaStream_t s);
// The chain weights of trsv_lu32_inv (WL, WU: chain_weights_elems(n) floats each):
// W_b = D_b^-1 L_{b,b-1}, V_b = D_b^-1 L_{b,b-2} (and the same with U) over the 128-row blocks,
// FP16 scaled, in the order the chain's tensor-core products read them.  (WL = WU = nullptr: the
// solve without the chain.)
size_t chain_weights_elems(int n);
// The poll limit of every triangular-solve wait (device constant; default 4,194,304).
cudaError_t set_wait_limit(unsigned spins);
cudaError_t chain_weights32(const float* LU, long lda, const float* DL, const float* DU, int n, float* WL, float* WU,
                            cudaStream_t s);
// Sets *d_status = kNotFinite if any of the n x nrhs entries is NaN or Inf.
cudaError_t check_finite(const double* X, long ldx, int n, int nrhs, int* d_status, cudaStream_t s);

// adjoint.cu ---------------------------------------------------------------------------------
// Pair integrals' adjoint: lam, fs [t][C][3] (adjoint vectors and solutions per column), col_out[c]
// = the result (0..K-1) column c belongs to.  xbar (n x 3K): d/d incenter; qbar (n x 10K): d/d
// corners (9) and d/d corrected area, summed over all pairs (the weight is -sum_c lam_c F_c^T).
size_t pair_adjoint_scratch_bytes(int n, int K);
cudaError_t launch_pair_adjoint(const DevMesh& m, int K, const double* lam, const double* fs, int C,
                                const int* col_out, double* xbar, double* qbar, void* scratch, cudaStream_t s);
// Per-triangle geometry's adjoint: cot [t][K][16] (self9, incenter, raw area, unit normal) -> vbar [t][K][9].
cudaError_t launch_tri_adjoint(const DevMesh& m, int K, const double* cot, double* vbar, cudaStream_t s);

// tc_gemm.cu ---------------------------------------------------------------------------------
// BF16 operand copies for the tensor-core GEMM: At (m x k row-major) from A (m x k column-major
// FP32), Bt (k x n column-major) from B (k x n column-major FP32).
cudaError_t cast_transpose_bf16(const float* A, long lda, int m, int k, void* At, long lda_t, cudaStream_t s);
cudaError_t cast_bf16(const float* B, long ldb, int k, int n, void* Bt, long ldb_t, cudaStream_t s);
// C (FP32, column-major) -= A B with A given as At (m x k row-major BF16) and B as Bt (k x n
// column-major BF16); tcgen05 kind::f16, FP32 accumulation in TMEM.
cudaError_t gemm_bf16_tc_minus(int m, int n, int k, const void* At, long lda_t, const void* Bt, long ldb_t, float* C,
                               long ldc, int* d_status, cudaStream_t s);
// Tensor maps (two opaque 128-byte CUtensorMap objects) over whole operand buffers, built once; and
// the GEMM on them (A = leading m rows of the A buffer, B = leading n rows of the B buffer).
constexpr int kTensorMapBytes = 128;
cudaError_t tc_gemm_prepare();  // kernel attributes, once, before any capture
bool tc_operand_maps(const void* At, int rows_a, long lda_t, const void* Bt, int rows_b, long ldb_t, void* map_a,
                     void* map_b);
// stamp (optional, here and below): 2 words per launch, set to [~0, 0] by stamps_reset; the kernel
// leaves its first start and last end (global timer, ns) there
cudaError_t gemm_bf16_tc_minus_maps(int m, int n, int k, const void* map_a, const void* map_b, float* C, long ldc,
                                    int* d_status, cudaStream_t s, unsigned long long* stamp = nullptr);
cudaError_t stamps_reset(unsigned long long* stamps, int slots, cudaStream_t s);
// Maps over whole-matrix BF16 mirrors (Am row-major, Bm column-major, n x n, ld ldm) and the GEMM on
// blocks of them named by position (A at rows a_row.., columns a_k..; B at columns b_row..,
// rows b_k..).
bool tc_mirror_maps(const void* Am, const void* Bm, int n, long ldm, void* map_a, void* map_b);
// Panel products of the FP32 LU on the tensor cores (TF32 operands, FP32 accumulation), a 128 x 128
// operand R against a panel P of len rows or columns (tc_gemm.cu, k_panel_tf32):
//   left:  X (h x len) := R P, or -= R P (sub);   right: X (len x h) := P R, or -= P R (sub)
// (h <= 128; subtracting, h <= 256: two row groups of R, grid.y)
// maps: kPanelMaps tensor maps (kPanelMaps kTensorMapBytes, built by tc_panel_maps) over the
// diagonal-block inverses dl, du (128 x 128 column-major each, one per 128 rows) and the factor
// (n x n, ld; kMapC: the BF16 GEMM's C tiles); map_r, map_p pick R's and P's.  The left form reads R through an MN-major map (kMapDL, kMapMN) and P through a K-major
// one (kMapK); the right form R K-major (kMapDU, kMapK) and P MN-major (kMapMN).  R's block starts at
// map coordinates (rx0, ry0) (inner, outer), P's at (px0, py0); rx0, px0 multiples of 4.  The assigning
// form writes the BF16 mirror too (mir: left column-major, right row-major; null: none).
constexpr int kMapDL = 0, kMapDU = 1, kMapK = 2, kMapMN = 3, kMapC = 4, kPanelMaps = 5;
bool tc_panel_maps(const float* lu32, int n, long ld, const float* dl, const float* du, void* maps);
// X sits at row xr0, column xc0 of the factor (multiples of 4; the mirror's position coordinate --
// xr0 left, xc0 right -- of 8); whole 128 x 128 tiles are stored by TMA through mirror_maps (two
// tensor maps from tc_mirror_store_maps: [0] the column-major mirror, [1] the row-major one), which
// must be given when mir is.
bool tc_mirror_store_maps(const void* Am, const void* Bm, int n, long ldm, void* maps);
cudaError_t panel_tf32(bool left, bool sub, const void* maps, int map_r, int map_p, const void* mirror_maps, int rx0,
                       int ry0, int px0, int py0, int h, int len, float* X, long ldx, int xr0, int xc0, void* mir,
                       long ldm, int* d_status, cudaStream_t s, unsigned long long* stamp);
// map_c (optional): a tensor map over C's FP32 matrix (tc_panel_maps' kMapC) with C at (c_row, c_col)
// of it (c_row a multiple of 4): products of at most 8 K tiles then load and store whole C tiles by
// TMA through shared memory.
// The 256-deep triangular-solve leaf (k_leaf256_tf32): the inverses of 256 x 256 diagonal blocks,
// column-major, one per slot (256 x 256 floats each; slot = the block's first row / 128), from
// k_combine256 -- left [[D1, 0], [F, D2]] in dl256, right [[E1, G], [0, E2]] in du256; t_maps: two
// tensor maps over them (tc_leaf256_maps).  Left: rows [kd, kd + h) x columns [p0, p0 + len) := Tinv
// times that block; right: rows [p0, p0 + len) x columns [kd, kd + h) := that block times Tinv; in
// place, with the BF16 mirror as panel_tf32's (kd, p0 multiples of 8; h <= 256).
bool tc_leaf256_maps(const float* dl256, const float* du256, int slots, void* maps);
// (mixed.cu) the 256 x 256 inverses of the diagonal block at (k0, k0) into slot k0 / 128 of TL, TU
cudaError_t combine256(const float* LU, long lda, int k0, const float* DL, const float* DU, float* TL, float* TU,
                       cudaStream_t s);
cudaError_t leaf256_tf32(bool left, const void* maps, const void* t_maps, const void* mirror_maps, int slot, int kd,
                         int p0, int h, int len, float* X, long ldx, void* mir, long ldm, int* d_status, cudaStream_t s,
                         unsigned long long* stamp);
cudaError_t gemm_bf16_tc_minus_at(int m, int n, int k, const void* map_a, int a_row, int a_k, const void* map_b,
                                  int b_row, int b_k, float* C, long ldc, int* d_status, cudaStream_t s,
                                  unsigned long long* stamp = nullptr, const void* map_c = nullptr, int c_row = 0,
                                  int c_col = 0);

}  // namespace bgpu
