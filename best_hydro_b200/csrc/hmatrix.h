// The hierarchical-matrix path for meshes whose dense GR does not fit in HBM (internal interface of
// libbestgpu).  The reference's answer to large N is its H-matrix with GMRES (hmatrix/src/hmatrix.cpp,
// cluster.cpp, gmres.cpp, driven by bhm_build/bhm_solve in hmatrix/src/api.cpp:582-771); this is the
// same decomposition built for the B200: the cluster tree and block partition on the host, every
// block filled on the device by the exact pair kernel (near blocks dense, far blocks by batched
// cross approximation), products and the block-Jacobi preconditioner as device kernels, restarted
// FP64 GMRES over all right-hand sides at once.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "bgpu_internal.h"

namespace bgpu {

// Cluster tree over the triangles and the partition of GR into blocks (host only).
struct HPlan {
  struct Cluster {
    int beg = 0, cnt = 0, level = 0;
    int son0 = -1;  // sons son0, son0 + 1; -1 for a leaf
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // bounding box of the corners
  };
  int n = 0, depth = 0;
  std::vector<int> perm;        // tree position -> triangle
  std::vector<Cluster> cl;      // cl[0] is the root
  std::vector<int> leaves;      // cluster ids of the leaves, in tree order
  struct Block {
    int t = 0, s = 0;           // row (target) and column (source) clusters
    bool lowrank = false;       // admissible and cheaper as a cross approximation than dense
    bool admissible = false;
  };
  std::vector<Block> blocks;
};

// Median-split cluster tree (hmatrix/src/cluster.cpp:10-113): depth the smallest with
// ceil(n / 2^depth) <= leaf, every cluster split at the median of its incenters along the incenters'
// longest extent (ties by triangle index), boxes over the corners; blocks from the root pair down,
// a pair admissible when min(diam) <= eta dist (cluster.cpp:115-117, hmatrix.cpp:26-53).  geo: n x
// kGeoStride (corners), xc: n x kXcStride (incenters).  An admissible block is low-rank when its
// cross approximation of at most kmax terms takes fewer entries than the block.
HPlan hplan_build(int n, const double* geo, const double* xc, int leaf, double eta, int kmax);

struct HReport {
  int iterations = 0;   // GMRES steps (all right-hand sides in lockstep)
  int restarts = 0;
  double relres = 0.0;  // largest true relative residual ||b - (H + deflation) x|| / ||b||
};

class HMatrixSolver {
 public:
  HMatrixSolver();
  ~HMatrixSolver();
  HMatrixSolver(const HMatrixSolver&) = delete;
  HMatrixSolver& operator=(const HMatrixSolver&) = delete;
  // Plans and fills the H-matrix of the mesh at relative accuracy eps, adds nothing for the deflation
  // (applied in every product as its low-rank term) and factors the block-Jacobi preconditioner.
  // Throws std::runtime_error on failure.
  void build(const DevMesh& m, const DevDeflation& d, int ndef, double eps, cudaStream_t s);
  // y = (H + deflation) x for nrhs columns (original triangle order, 3n rows).
  void matvec(int nrhs, const double* d_x, long ldx, double* d_y, long ldy, cudaStream_t s);
  // Solves in place by GMRES to a relative residual of 0.1 eps; throws when it does not converge.
  void solve(int nrhs, double* d_b, long ldb, cudaStream_t s, HReport* rep);
  // n, leaves, dense blocks, low-rank blocks, dense entries, low-rank entries (at their ranks), mean
  // rank, largest rank, blocks that reached kmax, fill ms, cross-approximation ms, preconditioner
  // ms, last solve's GMRES steps, its relative residual, device bytes held
  std::vector<double> stats() const;
  void set_options(int leaf, double eta, int kmax);

 private:
  struct Impl;
  Impl* p_;
};

}  // namespace bgpu
