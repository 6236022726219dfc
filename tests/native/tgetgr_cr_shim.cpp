// Test shim: the oracle's C restatement of TGETGR (oracle/tgetgr.c) compiled with correctly rounded
// acos/sin/cos/log (best_hydro_b200/csrc/ddmath.cuh) in place of glibc's.  With glibc's functions the
// restatement equals the reference bit for bit; with these, it must equal the GPU's entries bit for
// bit.  The difference between the two is exactly glibc's not-correctly-rounded results.
//
// Built twice (tests/crshim.py):
//   default            the correctly rounded restatement (orc_cr_*), OpenMP over target rows
//   -DBGPU_FN_PROBE    glibc's functions as the reference calls them, each call also evaluated
//                      correctly rounded; orc_pr_fn_misrounds counts, per triangle pair, the calls
//                      where glibc's result is not the correctly rounded one (single-threaded)
#include <cmath>
#include <cstdint>
#include <cstddef>

#include "../../best_hydro_b200/csrc/ddmath.cuh"

#ifdef BGPU_FN_PROBE
static long g_fn_mis = 0;
static inline void pr_count(double a, double b) {
  if (a != b && !(a != a && b != b)) ++g_fn_mis;
}
static inline double pr_log(double x) {
  const double a = std::log(x);
  pr_count(a, bgpu::dd::cr_log_tab(x, bgpu::dd::kLogTab));
  return a;
}
static inline double pr_acos(double x) {
  const double a = std::acos(x);
  pr_count(a, bgpu::dd::cr_acos(x));
  return a;
}
static inline double pr_sin(double x) {
  const double a = std::sin(x);
  pr_count(a, bgpu::dd::cr_sin(x));
  return a;
}
static inline double pr_cos(double x) {
  const double a = std::cos(x);
  pr_count(a, bgpu::dd::cr_cos(x));
  return a;
}
#define acos(x) pr_acos(x)
#define sin(x) pr_sin(x)
#define cos(x) pr_cos(x)
#define log(x) pr_log(x)
#define orc_self_blocks orc_pr_self_blocks
#define orc_gr_block orc_pr_gr_block
#define orc_diag_mean orc_pr_diag_mean
#define orc_deflate orc_pr_deflate
#define orc_ulp_hist orc_pr_ulp_hist
#else
#define acos(x) bgpu::dd::cr_acos(x)
#define sin(x) bgpu::dd::cr_sin(x)
#define cos(x) bgpu::dd::cr_cos(x)
#define log(x) bgpu::dd::cr_log_tab(x, bgpu::dd::kLogTab)
#define orc_self_blocks orc_cr_self_blocks
#define orc_gr_block orc_cr_gr_block
#define orc_diag_mean orc_cr_diag_mean
#define orc_deflate orc_cr_deflate
#define orc_ulp_hist orc_cr_ulp_hist
#endif

extern "C" {
#include "../../oracle/tgetgr.c"
}

#ifdef BGPU_FN_PROBE
extern "C" {
// For each triangle pair (n1[k], n2[k]): the number of acos/sin/cos/log calls of its 3x3 block where
// glibc's result differs from the correctly rounded one.  A self block (n1 == n2) is recomputed from
// its own triangle.  x: the reference's incenters (n x 3 column-major).
void orc_pr_fn_misrounds(int n, const double* v1, const double* v2, const double* v3, const double* area,
                         double afac, double cg, const double* x, long npairs, const int* n1, const int* n2,
                         long* counts) {
  double blk[9], tv[9], tx[3], t9[9];
  for (long k = 0; k < npairs; ++k) {
    g_fn_mis = 0;
    if (n1[k] == n2[k]) {
      const int t = n1[k];
      for (int c = 0; c < 3; ++c) {
        tv[c] = v1[(size_t)c * n + t];
        tv[3 + c] = v2[(size_t)c * n + t];
        tv[6 + c] = v3[(size_t)c * n + t];
      }
      orc_pr_self_blocks(1, tv, tv + 3, tv + 6, afac, cg, tx, t9);
    } else {
      orc_pr_gr_block(n, v1, v2, v3, area, cg, x, t9, n1[k], n1[k] + 1, n2[k], n2[k] + 1, blk, 3);
    }
    counts[k] = g_fn_mis;
  }
}
}
#endif
