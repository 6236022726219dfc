/* best_driver.h -- the host side of BEST around the solver seam, in C++ (libbestgpu).
 *
 * BEST's Fortran driver (best/best.f) does this work when it links libbestgpu; these functions let a
 * caller without Fortran run the same program: they restate the driver's set-up and post-processing
 * and reach the GPU only through the bhm_* seam.  Arrays are column-major like BEST's.
 */
#ifndef BEST_DRIVER_H
#define BEST_DRIVER_H

#ifdef __cplusplus
extern "C" {
#endif

/* best/best.f:261-337: tri holds 9 coordinates per triangle as read (row t: v1 v2 v3); returns
 * BEST's V1, V2, V3 (n x 3 column-major, centred), the corrected areas, AFAC, the total area, the
 * centroid, COMPON's surface labels (1-based), the number of surfaces and open edges, and NDEF. */
int bgpu_best_setup(int n, const double *tri, int iarea, double truearea, double *v1, double *v2, double *v3,
                    double *area, double *afac, double *totarea, double *centroid, int *icomp, int *ncomp,
                    int *nopen, int *ndef);

/* best/best.f:384-404 and DEFGAM (best/compon.f90:185-197): XMU (3n) and GDEF (ndef) from DIAGM. */
int bgpu_best_deflation(int n, const double *v1, const double *v2, const double *v3, const double *area, int ndef,
                        const int *icomp, double diagm, double *xmu, double *gdef);

/* best/difco.f:28-44: the six right-hand sides (3n x 6) from the incenters x (n x 3). */
void bgpu_best_rhs6(int n, const double *x, double *b);

/* best/visco.f:216-243: the five strain-flow right-hand sides (3n x 5). */
void bgpu_best_strain5(int n, const double *x, double *v);

/* best/difco.f:53-401 on the six solutions b6.  out (60 doubles): Dtt, Dtr, Drr (3x3 row-major),
 * urc, udr (3), Ktt, Krt and Krr at the centre of resistance (3x3 row-major). */
int bgpu_best_difco(int n, const double *x, const double *area, double cg, const double *b6, double *out);

/* best/visco.f:24-213: out[0] = CHI', out[1..3] = the viscosity centre (with icov = 1). */
int bgpu_best_visco(int n, const double *x, const double *area, double cg, int icov, const double *v5,
                    const double *b6, double *out);

/* best/output.f:96-130: out[0] 1/3 Tr Dtt (1/A), out[1] 1/3 Tr Drr (1/A^3), out[2] D_t (cm^2/s),
 * out[3] D_r (1/s), from bgpu_best_difco's tensors. */
void bgpu_best_traces(const double *tensors, double *out);

/* The linear extrapolation in 1/N of a series of results (BEST's workflow with rcoal, best/best.f:154-157,
 * README.md:12-16): the least-squares line y = y0 + slope / N through (1/n[i], y[i]), i < count
 * (count >= 2).  Returns y0 (the value at an infinite number of triangles); *slope may be NULL. */
double bgpu_best_extrapolate(int count, const int *n, const double *y, double *slope);

/* The whole program (best/best.f:184-510 through the seam, as with -hm): reads the mesh file, solves,
 * writes <infile><flags>.be and .log.  precision: 0 FP64 LU, 1 mixed, 2 H-matrix, -1 BEST's rule.  results
 * (may be NULL, 68 doubles): bgpu_best_difco's 60, then CHI', Dx, Dy, Dz, D_t, D_r, CHI, ETA. */
int bgpu_best_run(const char *infile, int iarea, int cg_zero, int ivisco, int icov, double wm, int precision,
                  double *results);

#ifdef __cplusplus
}
#endif

#endif
