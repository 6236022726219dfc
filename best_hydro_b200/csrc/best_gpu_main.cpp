// best_gpu: BEST's command line (best/input.f:26-68) on the GPU backend, for machines without a
// Fortran compiler.  best_gpu -f file [-na] [-p] [-v] [-vc] [-mw W] [-fp64 | -mixed | -hm]
// (-hm: the H-matrix path at BEST's default accuracy 1e-4, as BEST's own -hm flag selects its H-matrix
// solver; without a flag, meshes whose dense matrix does not fit on the GPU take it by themselves)
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/best_driver.h"

int main(int argc, char** argv) {
  const char* file = nullptr;
  int iarea = 1, cgz = 0, iv = 0, icov = 0, prec = -1;
  double wm = 0;
  for (int k = 1; k < argc; ++k) {
    if (!std::strcmp(argv[k], "-f") && k + 1 < argc) file = argv[++k];
    else if (!std::strcmp(argv[k], "-na")) iarea = 0;
    else if (!std::strcmp(argv[k], "-p")) cgz = 1;
    else if (!std::strcmp(argv[k], "-v")) iv = 1;
    else if (!std::strcmp(argv[k], "-vc")) iv = icov = 1;
    else if (!std::strcmp(argv[k], "-mw") && k + 1 < argc) wm = std::atof(argv[++k]);
    else if (!std::strcmp(argv[k], "-fp64")) prec = 0;
    else if (!std::strcmp(argv[k], "-mixed")) prec = 1;
    else if (!std::strcmp(argv[k], "-hm")) prec = 2;
  }
  if (!file) {
    std::printf("Usage : best_gpu -f input_filename [-na] [-p] [-v] [-vc] [-mw W] [-fp64 | -mixed | -hm]\n");
    return 0;
  }
  const int rc = bgpu_best_run(file, iarea, cgz, iv, icov, wm, prec, nullptr);
  if (rc != 0) std::printf("BEST: the GPU solve failed; see the .log file\n");
  return rc != 0 ? 1 : 0;
}
