/* best_gpu.h -- extensions of libbestgpu beyond BEST's nine-function seam (best_hmatrix.h).
 *
 * Precision control, timings, device-pointer entry points for callers that keep their data on the
 * GPU, and the raw FP64 factor/solve kernels with LAPACK semantics.  The reference has no GPU code,
 * so none of these replaces a reference function one for one; each names the reference routine
 * whose semantics it follows.  Every int-returning function returns 0 on success, or nonzero after
 * queuing a message for bhm_log_line.  Device pointers must be 16-byte aligned and leading
 * dimensions even.  The library works on its own non-blocking stream (bgpu_stream): data written on
 * other streams must be complete before a call, and each call has finished with its data on return.
 */
#ifndef BEST_GPU_H
#define BEST_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Factorisation precisions for bhm_build. */
enum {
  BGPU_FP64 = 0,    /* FP64 LU with partial pivoting (the plain path) */
  BGPU_MIXED = 1,   /* reduced-precision tensor-core LU + FP64 GMRES refinement */
  BGPU_HMATRIX = 2  /* H-matrix (dense near field, low-rank far field) + FP64 GMRES: N beyond HBM */
};

/* Overrides the precision bhm_build derives from direct/single (-1: back to that rule).  Without an
 * override, bhm_build takes BGPU_HMATRIX by itself when the dense GR of the chosen path does not fit
 * in the GPU's free memory (logged). */
int bgpu_set_precision(int mode);

/* The precision of the last bhm_build. */
int bgpu_precision(void);

/* Refinement of the mixed path: at most max_restarts GMRES restarts (each starting from the true
 * FP64 residual) of krylov <= 16 vectors; defaults 8 and 10.  When the refinement does not reach its
 * tolerance, bhm_solve factors the kept FP64 matrix on the GPU and solves with it instead (logged). */
int bgpu_set_refinement(int max_restarts, int krylov);

/* The H-matrix path (the GPU counterpart of the reference's H-matrix solver, hmatrix/src/api.cpp:582-771,
 * selected by BEST's -hm or N > 10,000 there; here by bgpu_set_precision(BGPU_HMATRIX) or when the dense
 * GR does not fit).  bhm_build's eps is the relative accuracy of the far-field blocks (BEST's -he,
 * default 1e-4); bhm_solve runs GMRES(30) to a relative residual of 0.1 eps (hmatrix/src/api.cpp:39-41).
 * Every entry the H-matrix evaluates equals bhm_entries' entry bit for bit; the deflation is applied as
 * a low-rank term of every product (api.cpp:641-646).
 *
 * Settings of later builds: leaf clusters of at most `leaf` triangles (8..128; default 128), the
 * admissibility eta (default 2.0, cluster.cpp:115-117), at most kmax (multiple of 3, <= 120; default
 * 90) terms per low-rank block. */
int bgpu_hmatrix_set_options(int leaf, double eta, int kmax);

/* Figures of the last H-matrix build and solve, up to len of: n, leaves, dense blocks, low-rank blocks,
 * dense entries, low-rank entries (at their ranks), mean rank, largest rank, blocks that reached kmax,
 * fill ms, cross-approximation ms, preconditioner ms, GMRES steps of the last solve, its largest
 * relative residual, device bytes held. */
int bgpu_hmatrix_stats(double *out, int len);

/* y = (H + deflation) x on device data (3n x nrhs, leading dimensions ldx, ldy >= 3n), original
 * triangle order: the product GMRES uses. */
int bgpu_hmatrix_matvec_device(int nrhs, const double *d_x, int ldx, double *d_y, int ldy);

/* The H-matrix's cluster tree and block partition alone, on the host (no GPU used): x the incenters
 * and v1, v2, v3 the corners (n x 3 column-major, as bhm_create takes them).  perm[k] receives the
 * triangle at tree position k (0-based); counts[0..4]: depth, leaves, dense blocks, low-rank blocks,
 * admissible blocks. */
int bgpu_hmatrix_plan(int n, const double *x, const double *v1, const double *v2, const double *v3, int leaf,
                      double eta, int kmax, int *perm, int *counts);

/* Stage times of the last calls in milliseconds, measured with CUDA events on the library's
 * stream: ms[0] self blocks + incenters (bhm_create), ms[1] assembly + deflation, ms[2] LU,
 * ms[3] solve (last bhm_solve or bgpu_solve_device), ms[4] bhm_build total, ms[5] refinement
 * iterations of the last solve (count, as a double), ms[6] relative residual of the last solve.
 * Returns the number of values written (at most len). */
int bgpu_timings(double *ms, int len);

/* The library's CUDA stream (a cudaStream_t), for callers that order their own work after it. */
void *bgpu_stream(void);

/* bhm_solve for right-hand sides already on the GPU: d_b is 3n x nrhs with leading dimension ldb. */
int bgpu_solve_device(int nrhs, double *d_b, int ldb);

/* LAPACK dgetrf semantics on a caller's device matrix (best/best.f:444): d_a (n x n, column-major,
 * lda) is overwritten by L and U, d_ipiv receives the 1-based interchanges, *info (host) the first
 * exactly-zero pivot (1-based) or 0. */
int bgpu_dgetrf_device(int n, double *d_a, int lda, int *d_ipiv, int *info);

/* LAPACK dgetrs('N') semantics on device data (best/besolve.f90:133): solves with the factors of
 * bgpu_dgetrf_device for nrhs <= 16 right-hand sides d_b (n x nrhs, ldb), in place. */
int bgpu_dgetrs_device(int n, int nrhs, const double *d_a, int lda, const int *d_ipiv, double *d_b, int ldb);

/* The solve of bgpu_dgetrs_device for callers that cannot allocate GPU memory.  It calls no
 * cudaMalloc, cudaFree or other allocating routine: an application that owns all device memory
 * through its own pool allocator, or that must not let a library allocate behind its back, can still
 * solve with the factors.  Its scratch (readiness flags, the permuted right-hand sides, the
 * permutation, a status word) is a fixed 16 MiB array in the library's device image, which every GPU
 * that uses it holds until the process exits; that bounds the order: n * (8 * 16 + 4) bytes plus a
 * few KB must fit, i.e. n <= about 127,000 (larger n is rejected with a message).
 * The array gets its device memory when the library's module is loaded on the device, which under
 * CUDA's default lazy loading happens at the first call, not when the library is loaded: make a
 * first call -- n = 0 is a warm-up that only looks the array up and runs the solve's kernels once on
 * a 1 x 1 system inside it -- on each device, with that device current, before the application's
 * allocator reserves the memory, and before any stream capture.  Later calls touch no memory beyond
 * the array and their arguments.
 * stream: a cudaStream_t (NULL for the default stream); the call waits for the solve on it to finish
 * and returns 0, or nonzero after a message.  Every call uses the same array, which keeps the last
 * call's contents: calls that overlap on the GPU (other threads, other streams of the same device)
 * race and must be serialised by the caller.  No reference counterpart: the reference has no GPU
 * code. */
int bgpu_dgetrs_noalloc(int n, int nrhs, const double *d_a, int lda, const int *d_ipiv, double *d_b, int ldb,
                        void *stream);

/* C(m x n) -= A(m x k) B(k x n), FP64, column-major device matrices: the LU's trailing update. */
int bgpu_dgemm_minus_device(int m, int n, int k, const double *d_a, int lda, const double *d_b, int ldb,
                            double *d_c, int ldc);

/* C(m x n) -= A(m x k) B(k x n) with A, B rounded to BF16 and FP32 accumulation on the tcgen05
 * tensor cores (column-major FP32 device matrices): the mixed-precision LU's update. */
int bgpu_gemm_bf16_minus_device(int m, int n, int k, const float *d_a, int lda, const float *d_b, int ldb, float *d_c,
                                int ldc);

/* ---- Input set-up on the GPU (BEST's driver does it on the host: best/best.f:261-337 and COMPON,
 * best/compon.f90:19-116; the deflation, best/best.f:384-404 and DEFGAM, compon.f90:185-197) ------
 * bgpu_create_from_triangles takes the triangles as read (tri: n x 9, row t = v1 v2 v3, host memory)
 * and does on the device what BEST does before bhm_create -- centroid shift, areas, the area
 * correction (iarea, truearea), COMPON's surfaces and open edges, NDEF -- and then what bhm_create
 * does.  info (5 doubles, may be NULL): AFAC, total area, centroid; counts (3 ints, may be NULL):
 * surfaces, open edges, NDEF.  Every value equals bgpu_best_setup's bit for bit (the sums are taken
 * in BEST's order).  bgpu_build_prepared then forms XMU and GDEF from DIAGM on the device and
 * builds as bhm_build does with them (eps, direct, single as there).  bgpu_prepared_arrays copies
 * the set-up out (any pointer may be NULL): V1, V2, V3 (n x 3 column-major, centred), corrected
 * areas, surface labels, and after bgpu_build_prepared XMU (3n) and GDEF (NDEF). */
int bgpu_create_from_triangles(int n, const double *tri, int iarea, double truearea, double cg, double *info,
                               int *counts);
int bgpu_build_prepared(double eps, int direct, int single, int nrhs);
int bgpu_prepared_arrays(double *v1, double *v2, double *v3, double *area, int *icomp, double *xmu, double *gdef);

/* Every wait of the triangular solves (a block row waiting for the rows it depends on) polls at
 * most `spins` times, then the kernel records a timeout and returns, and the call fails with a
 * message instead of hanging: 4,194,304 polls by default.  0 makes any wait that is not satisfied at
 * once give up -- for tests of that failure path.  The solver stays usable afterwards. */
int bgpu_set_wait_limit(unsigned spins);

/* The mixed-precision LU's diagonal leaf (FP32, device memory): the h x h block d_a (h <= 128,
 * column-major, lda) factored without pivoting in place (unit L below, U on and above the diagonal),
 * L^-1 into d_linv and U^-1 into d_uinv (128 x 128 column-major each, zero outside h x h).  A zero
 * or non-finite pivot is an error. */
int bgpu_lu32_leaf_device(int h, float *d_a, int lda, float *d_linv, float *d_uinv);

/* The mixed-precision LU's triangular-solve leaf on the tensor cores (TF32 operands, FP32
 * accumulation; device memory).  d_a: the n x n FP32 factor (column-major, lda a multiple of 4);
 * d_linv, d_uinv: the diagonal blocks' inverses, 128 x 128 column-major each, one per 128 rows
 * (block b at b * 16384), zero outside the block's h x h.  left != 0: rows [kd, kd + h) x columns
 * [p0, p0 + len) := L_kd^-1 times that block (d_linv's block kd / 128); left == 0: rows [p0, p0 + len) x
 * columns [kd, kd + h) := that block times U_kd^-1 (d_uinv's).  In place; with d_mirror (BF16,
 * n x n, ldm) the result's BF16 copy goes to the same positions of d_mirror, column-major for the
 * left leaf and row-major (element (i, j) at i * ldm + j) for the right one (ldm a multiple of 8).
 * kd and p0 multiples of 32, h <= 128. */
int bgpu_trsm_leaf_device(int left, int n, float *d_a, int lda, const float *d_linv, const float *d_uinv, int kd,
                          int p0, int h, int len, void *d_mirror, int ldm);

/* The mixed-precision LU's 256-deep triangular-solve leaf (TF32 tensor cores; device memory): the
 * inverse of the 256 x 256 diagonal block at (kd, kd) of the n x n FP32 factor d_a (unit lower L and
 * upper U packed, column-major, lda a multiple of 4) is formed from the inverses of its two 128-blocks
 * (d_linv, d_uinv as bgpu_trsm_leaf_device's) and the off-diagonal blocks L21, U12 of d_a, then left
 * != 0: rows [kd, kd + 256) x columns [p0, p0 + len) := L^-1 times that block; left == 0: rows
 * [p0, p0 + len) x columns [kd, kd + 256) := that block times U^-1; in place, with the BF16 mirror as
 * bgpu_trsm_leaf_device's.  kd a multiple of 128, p0 of 32. */
int bgpu_trsm_leaf256_device(int left, int n, float *d_a, int lda, const float *d_linv, const float *d_uinv, int kd,
                             int p0, int len, void *d_mirror, int ldm);

/* The mixed-precision LU's K = 128 update on the tensor cores (TF32 operands, FP32 accumulation;
 * device memory): in the n x n FP32 matrix d_a (column-major, lda a multiple of 4), the m x nc block
 * at (cr, cc) -= the m x 128 block at (ar, ac) times the 128 x nc block at (br, bc), with m or nc at
 * most 256 and ar, br, cr multiples of 4.  The blocks may lie anywhere in the matrix but the result
 * block must not overlap the other two. */
int bgpu_panel_update_device(int n, float *d_a, int lda, int m, int nc, int ar, int ac, int br, int bc, int cr,
                             int cc);

/* Assembles GR rows of triangles [r0, r1) x columns of triangles [c0, c1) of the mesh given to
 * bhm_create into d_out (column-major, ldo), before deflation (best/tgetgr.f:33-173). */
int bgpu_assemble_device(int r0, int r1, int c0, int c1, double *d_out, int ldo);
/* The same block with the mixed-precision path's assembly: fewer FP64 operations (rsqrt, shared
 * reciprocals, FMA contraction); entries within a few ulp of bgpu_assemble_device's, not
 * bit-compatible with the reference. */
int bgpu_assemble_device_mixed(int r0, int r1, int c0, int c1, double *d_out, int ldo);

/* ---- Series of meshes (BEST's workflow of results extrapolated linearly in 1/N: rcoal makes a
 * series of triangulations of one surface, best/best.f:154-157, README.md:12-16) ---------------
 * Up to 16 meshes are assembled, factored (FP64 LU with partial pivoting, the plain path) and solved
 * together: one launch assembles all of them, and each step of the blocked LU runs as one launch per
 * kernel for every mesh at once; the whole build is captured once as a CUDA graph and replayed.
 * Each mesh's factors and solutions are those of factoring it alone (bhm_build with direct = 1).
 * Arrays of several meshes are concatenated: mesh i's block follows mesh i-1's, in the layout of
 * the single-mesh call (v1, v2, v3: n_i x 3 column-major; x: n_i x 3; xmu: 3 n_i; comp: n_i;
 * gdef: ndef_i values; b: 3 n_i x nrhs column-major). */

/* Copies the meshes (set-up done by the caller, as for bhm_create) and computes incenters and self
 * blocks.  n: triangles of each mesh; afac: each mesh's area correction factor. */
int bgpu_series_create(int count, const int *n, const double *v1, const double *v2, const double *v3,
                       const double *area, const double *afac, double cg);

/* The meshes' incenters (concatenated n_i x 3 blocks), as bhm_incenters. */
int bgpu_series_incenters(double *x);

/* BEST's mean of GR's diagonal for each mesh (count values), as bhm_diag_mean. */
int bgpu_series_diag_mean(double *dm);

/* Assembles every GR with its deflation (best/best.f:406-425) and factors it.  tune = 1 first runs
 * the build once with the DGEMM tile-shape autotuner on (its choices are logged and kept for the
 * process), then builds again from the tuned graph.  Nonzero on a zero pivot (the message names the
 * mesh), as bhm_build. */
int bgpu_series_build(const int *ndef, const double *gdef, const int *comp, const double *xmu, int tune);

/* Solves every mesh's system for nrhs right-hand sides in place (concatenated blocks). */
int bgpu_series_solve(int nrhs, double *b);

/* The precision of the next bgpu_series_build: BGPU_FP64 (default: the batched FP64 LU above, each
 * mesh's solution that of its single plain solve bit for bit) or BGPU_MIXED: every mesh's assembly
 * and BF16 tensor-core factorisation (the mixed path of bhm_build) enqueued on a stream of its own,
 * so the meshes' factorisations run side by side, and FP64 GMRES-IR solves to a relative residual of
 * 1e-12 (each mesh's solution that of its single mixed solve).  A mesh the unpivoted factorisation
 * cannot handle makes the build fall back to the FP64 series (logged). */
int bgpu_series_set_precision(int mode);

/* ms[0] last series build (graph replay), ms[1] the assembly of the last direct (tuning or
 * uncaptured) build, ms[2] last series solve, ms[3] the tuning pass (0 when not tuned).  Returns
 * the number of values written. */
int bgpu_series_timings(double *ms, int len);

void bgpu_series_destroy(void);

/* The DGEMM autotuner's choices so far as text, one line per size class (NUL-terminated in buf of
 * len bytes); returns the full length. */
int bgpu_autotune_table(char *buf, int len);

/* ---- Gradients (the adjoint method) --------------------------------------------------------
 * BEST's D_t and D_r (best/output.f:96-130) and [eta] (best/visco.f with icov = 0) of the mesh given
 * to bhm_create, and their gradients with respect to every corner coordinate of every triangle.  It
 * needs the FP64 LU of the last bhm_build, solves the 6 + 5 flows itself, solves the transposed
 * systems with the same factors, and recomputes GR's entries on the GPU (never stored) to contract
 * their derivatives.  The whole set-up is differentiated: the centroid shift (best.f:261-272), the
 * area correction AFAC (iarea = 1: TRUEAREA / the total area), the deflation (best.f:384-425) and the
 * self blocks.  wm: molecular weight ([eta] = CHI' 0.602214 / wm cm^3/g); wm <= 0 gives CHI' (A^3).
 * values[3]: D_t (cm^2/s), D_r (1/s), [eta].  grad (27 n doubles): for each result k, 9 n values
 * d values[k] / d(V1, V2, V3) (three n x 3 column-major blocks, per Angstrom, the coordinates as
 * read, before the centroid shift).  No reference counterpart: the reference has no derivatives. */
int bgpu_best_gradient(int iarea, double truearea, double wm, double *values, double *grad);

/* Kernel launches the library has issued since it was loaded. */
unsigned long long bgpu_launch_count(void);

/* Kernels whose launches can be timed live (CUDA events on the library's stream). */
enum {
  BGPU_KERNEL_LU_GEMM64 = 0, /* the FP64 LU's trailing-update GEMM (DMMA) */
  BGPU_KERNEL_TC_GEMM = 1    /* the mixed LU's tcgen05 BF16 GEMM (every update of the factorisation) */
};

/* Returns, for `kernel`, the launches recorded since the last call, their summed device time (ms) and
 * their algorithmic work (flops), then turns recording on (enable = 1) or off (0).  While the mixed
 * LU's GEMM is recorded, its factorisation is launched directly instead of replayed from its graph. */
int bgpu_kernel_stats(int kernel, int enable, int *launches, double *ms, double *work);

#ifdef __cplusplus
}
#endif

#endif
