// Test shim: the oracle's C restatement of TGETGR (oracle/tgetgr.c) compiled with correctly rounded
// acos/sin/cos/log (best_hydro_b200/csrc/ddmath.cuh) in place of glibc's.  With glibc's functions the
// restatement equals the reference bit for bit; with these, it must equal the GPU's self blocks bit
// for bit.  The difference between the two is exactly glibc's not-correctly-rounded results.
#include <cmath>
#include <cstdint>
#include <cstddef>

#include "../../best_hydro_b200/csrc/ddmath.cuh"

#define acos(x) bgpu::dd::cr_acos(x)
#define sin(x) bgpu::dd::cr_sin(x)
#define cos(x) bgpu::dd::cr_cos(x)
#define log(x) bgpu::dd::cr_log(x)
#define orc_self_blocks orc_cr_self_blocks
#define orc_gr_block orc_cr_gr_block
#define orc_diag_mean orc_cr_diag_mean
#define orc_deflate orc_cr_deflate
#define orc_ulp_hist orc_cr_ulp_hist

extern "C" {
#include "../../oracle/tgetgr.c"
}
