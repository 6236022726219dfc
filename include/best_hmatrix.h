/* best_hmatrix.h -- BEST's solver seam, served by the B200 dense backend (libbestgpu).
 *
 * BEST (best/besolve.f90:48-89) binds these nine functions with bind(C) and calls them when it
 * runs its solver behind the C interface (-hm, or more than NHMAT = 10000 triangles with
 * bhm_available() != 0; best/best.f:202-205).  libbestgpu exports them with the same names,
 * signatures and conventions as the reference's H-matrix library, so linking it in place of that
 * library (reference Makefile HMATRIX switch, :54-63) changes no Fortran.  Behind the seam the
 * backend assembles the dense 3N x 3N matrix GR on the GPU (FP64, bit-compatible with TGETGR), adds
 * the normal-field deflation, factors it (FP64 LU, or a tensor-core LU refined to FP64 accuracy)
 * and solves.
 *
 * Conventions (as the reference's, hmatrix/best_hmatrix.h:12-15): one solver per process; calls
 * come from one host thread; unknown 3 n + a (from 0) is component a of the traction on triangle n;
 * arrays are owned by the caller and column-major; a nonzero return means a message was queued
 * for bhm_log_line.  No C++ exception crosses this interface.
 */
#ifndef BEST_HMATRIX_H
#define BEST_HMATRIX_H

#ifdef __cplusplus
extern "C" {
#endif

/* 1 when a CUDA device is usable, else 0 (replaces hmatrix/best_hmatrix.h:27; the Fortran stand-in
 * best/hmstub.f90:7-11 returns 0). */
int bhm_available(void);

/* Copies the triangulation to the GPU and computes the incenters and the exact self blocks
 * (replaces hmatrix/best_hmatrix.h:34-35, implemented in the reference at hmatrix/src/api.cpp:777-791).
 * v1, v2, v3: BEST's V1, V2, V3 (n x 3, column-major, after the centroid shift); area: the areas
 * after the area correction; afac: the correction factor; cg: 1, or 0 with -p.  threads is
 * accepted for compatibility and ignored.  Returns 0, or nonzero after queuing a message. */
int bhm_create(int n, const double *v1, const double *v2, const double *v3, const double *area, double afac,
               double cg, int threads);

/* The incenters as TGETGR computes them (best/tgetgr.f:36-52), n x 3 column-major
 * (replaces hmatrix/best_hmatrix.h:38; reference hmatrix/src/api.cpp:793-801). */
void bhm_incenters(double *x);

/* Entries of GR before deflation, rows i0 .. i0+m-1, columns j0 .. j0+nc-1, into a (column-major,
 * leading dimension lda), computed on the GPU (replaces hmatrix/best_hmatrix.h:42; reference
 * hmatrix/src/api.cpp:803-828). */
void bhm_entries(int i0, int m, int j0, int nc, double *a, int lda);

/* The mean of GR's diagonal, summed in BEST's order (best/best.f:401-403; replaces
 * hmatrix/best_hmatrix.h:45; reference hmatrix/src/api.cpp:830). */
double bhm_diag_mean(void);

/* Assembles GR + sum_k gdef[k] xmu_k xmu_k^T on the GPU and factors it (replaces
 * hmatrix/best_hmatrix.h:61-62; reference hmatrix/src/api.cpp:832-866; dense equivalent
 * best/best.f:351-468).  ndef, gdef, comp, xmu: the deflation of best/best.f:384-426 (comp[i] in
 * 1..ndef is the surface of triangle i; xmu has 3n entries).  The H-matrix controls are reread as
 * precision controls:
 *   direct = 1                  plain FP64 LU with partial pivoting (dgetrf semantics);
 *   direct = 0 (or single = 1)  tensor-core LU in reduced precision, each bhm_solve refined by
 *                               GMRES with FP64 residuals to a relative residual of 0.1 * eps
 *                               (FP64 LU when BEST_GPU_PRECISION=fp64);
 * eps_pre and nrhs are accepted and unused.  Returns 0, or nonzero after queuing a message (a zero
 * pivot: "U(i,i) = 0", the same condition as dgetrf's info > 0, best/best.f:458-468). */
int bhm_build(double eps, int direct, double eps_pre, int ndef, const double *gdef, const int *comp,
              const double *xmu, int single, int nrhs);

/* Solves GR x = b in place for nrhs right-hand sides (b is 3n x nrhs, column-major); replaces
 * hmatrix/best_hmatrix.h:66 (reference hmatrix/src/api.cpp:868-879) and dgetrs
 * (best/besolve.f90:132-133).  Returns 0, or nonzero after queuing a message (solution not finite,
 * refinement did not converge). */
int bhm_solve(int nrhs, double *b);

/* Copies the next queued message into buf (at most len characters, no terminating NUL) and returns
 * its length, or -1 when there is none (replaces hmatrix/best_hmatrix.h:70; reference
 * hmatrix/src/api.cpp:881-890). */
int bhm_log_line(char *buf, int len);

/* Frees everything on the host and the GPU (replaces hmatrix/best_hmatrix.h:73). */
void bhm_destroy(void);

#ifdef __cplusplus
}
#endif

#endif
