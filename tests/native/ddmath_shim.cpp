// Test shim: exposes the product's double-double math (best_hydro_b200/csrc/ddmath.cuh), compiled as
// host C++ with -ffp-contract=off, to the CPU tests through ctypes.
#include "../../best_hydro_b200/csrc/ddmath.cuh"

extern "C" {
void dd_log_v(int n, const double* x, double* y) { for (int i = 0; i < n; ++i) y[i] = bgpu::dd::cr_log(x[i]); }
void dd_sin_v(int n, const double* x, double* y) { for (int i = 0; i < n; ++i) y[i] = bgpu::dd::cr_sin(x[i]); }
void dd_cos_v(int n, const double* x, double* y) { for (int i = 0; i < n; ++i) y[i] = bgpu::dd::cr_cos(x[i]); }
void dd_acos_v(int n, const double* x, double* y) { for (int i = 0; i < n; ++i) y[i] = bgpu::dd::cr_acos(x[i]); }
void dd_log_tab_v(int n, const double* x, double* y) {
  for (int i = 0; i < n; ++i) y[i] = bgpu::dd::cr_log_tab(x[i], bgpu::dd::kLogTab);
}
// the fast phase's hi and lo, and the accurate phase's, for error measurements
void dd_log_fast_v(int n, const double* x, double* hi, double* lo) {
  for (int i = 0; i < n; ++i) {
    const bgpu::dd::DD y = bgpu::dd::log_fast_dd(x[i], bgpu::dd::kLogTab);
    hi[i] = y.hi;
    lo[i] = y.lo;
  }
}
void dd_log_acc_v(int n, const double* x, double* hi, double* lo) {
  for (int i = 0; i < n; ++i) {
    const bgpu::dd::DD y = bgpu::dd::log_dd(x[i]);
    hi[i] = y.hi;
    lo[i] = y.lo;
  }
}
void dd_ln2(double* hi, double* lo) {
  bgpu::dd::DD l = bgpu::dd::ln2();
  *hi = l.hi;
  *lo = l.lo;
}
}
