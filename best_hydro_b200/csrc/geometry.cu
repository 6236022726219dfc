// BEST's input set-up on the GPU: the mesh as read (n x 9 triangle corners) to the arrays the
// solver works on, without a host pass over the triangles.
//
//   k_centroid, k_center_area, k_area_total   best/best.f:261-315: centroid, centred corners,
//                                              areas, total area, area correction AFAC
//   k_vertex_insert, k_vertex_check,          COMPON, best/compon.f90:19-116: triangles that share
//   k_components, k_edge_insert, k_edge_open  a vertex (exact coordinates) form a surface, numbered
//                                              in the order of their first triangles; open edges
//                                              are edges not shared by exactly two triangles;
//                                              best.f:323-337: NDEF
//   k_xmu, k_gdef                             the normal-field deflation, best/best.f:384-404 and
//                                              DEFGAM best/compon.f90:185-197
//
// Compiled with -fmad=false, and every sum BEST accumulates in a DO loop (centroid, total area,
// |XMU|^2) is accumulated in that order by one thread (the terms themselves are formed in
// parallel), so the results equal the host restatement (driver.cpp) and the oracle bit for bit.
//
// Vertex identity is exact equality of the three centred coordinates (-0 equals +0), found by a
// hash table with a 64-bit hash; two different coordinate triples that collide in the hash are
// detected (every corner is compared with its slot's first corner) and the table is rebuilt with
// another seed.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "bgpu_internal.h"

namespace bgpu {
namespace {

constexpr unsigned long long kEmpty = ~0ull;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  // splitmix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number generators")
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long coord_bits(double x) {
  return (unsigned long long)__double_as_longlong(x + 0.0);  // -0 + 0 = +0
}

__device__ __forceinline__ unsigned long long vertex_hash(double x, double y, double z, unsigned long long seed) {
  unsigned long long h = mix64(seed ^ coord_bits(x));
  h = mix64(h ^ coord_bits(y));
  h = mix64(h ^ coord_bits(z));
  return h == kEmpty ? 0ull : h;
}

// corner k = 3 t + c of the centred mesh (geo: kGeoStride per triangle)
__device__ __forceinline__ void corner(const double* geo, int k, double& x, double& y, double& z) {
  const double* p = geo + (size_t)(k / 3) * kGeoStride + 3 * (k % 3);
  x = p[0];
  y = p[1];
  z = p[2];
}

// best.f:261-268: CEN(c) = (sum over triangles of (x1 + x2 + x3) / 3) / NAR, summed in order.  The
// terms are formed by the block, the running sum by one thread.
__global__ void k_centroid(int n, const double* __restrict__ tri, double* __restrict__ cen) {
  __shared__ double term[3][256];
  double s[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < n; b += 256) {
    const int t = b + threadIdx.x;
    if (t < n)
      for (int c = 0; c < 3; ++c)
        term[c][threadIdx.x] = (tri[9 * (size_t)t + c] + tri[9 * (size_t)t + 3 + c] + tri[9 * (size_t)t + 6 + c]) / 3;
    __syncthreads();
    if (threadIdx.x < 3) {
      const int c = threadIdx.x, m = min(256, n - b);
      for (int i = 0; i < m; ++i) s[c] = s[c] + term[c][i];
    }
    __syncthreads();
  }
  if (threadIdx.x < 3) cen[threadIdx.x] = s[threadIdx.x] / n;
}

// best.f:269-305: centred corners (geo and n x 3 column-major v1, v2, v3) and triangle areas
__global__ void k_center_area(int n, const double* __restrict__ tri, const double* __restrict__ cen,
                              double* __restrict__ geo, double* __restrict__ v, double* __restrict__ area) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double p[9];
  for (int q = 0; q < 9; ++q) p[q] = tri[9 * (size_t)t + q] - cen[q % 3];
  double* g = geo + (size_t)t * kGeoStride;
  for (int q = 0; q < 9; ++q) g[q] = p[q];
  g[10] = g[11] = 0.0;
  for (int cn = 0; cn < 3; ++cn)
    for (int c = 0; c < 3; ++c) v[(size_t)cn * 3 * n + (size_t)c * n + t] = p[3 * cn + c];
  const double v21x = p[3] - p[0], v21y = p[4] - p[1], v21z = p[5] - p[2];
  const double v31x = p[6] - p[0], v31y = p[7] - p[1], v31z = p[8] - p[2];
  const double a = v31y * v21z - v31z * v21y, b = v31z * v21x - v31x * v21z, c = v31x * v21y - v31y * v21x;
  area[t] = sqrt(a * a + b * b + c * c) * 0.5;
}

// best.f:306-315: total area (summed in order), AFAC = TRUEAREA / total with the area correction,
// and the corrected areas.  scal: [0] AFAC, [1] total area.
__global__ void k_area_total(int n, int iarea, double truearea, double* __restrict__ area, double* __restrict__ geo,
                             double* __restrict__ scal) {
  __shared__ double s_tot, s_afac;
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int t = 0; t < n; ++t) tot = tot + area[t];
    s_tot = tot;
    s_afac = iarea ? truearea / tot : 1.0;
    scal[0] = s_afac;
    scal[1] = tot;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const double a = iarea ? s_afac * area[t] : area[t];
    area[t] = a;
    geo[(size_t)t * kGeoStride + 9] = a;
  }
}

// COMPON, step 1: every corner into the vertex table (slot = first free or same-hash slot by
// linear probing); owner[slot] = the smallest corner index with that hash.
__global__ void k_vertex_insert(int n, const double* __restrict__ geo, unsigned long long seed,
                                unsigned long long* __restrict__ keys, int* __restrict__ owner, int* __restrict__ vslot,
                                unsigned mask, int* status) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * n) return;
  double x, y, z;
  corner(geo, k, x, y, z);
  const unsigned long long h = vertex_hash(x, y, z, seed);
  unsigned slot = (unsigned)h & mask;
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const unsigned long long prev = atomicCAS(keys + slot, kEmpty, h);
    if (prev == kEmpty || prev == h) {
      atomicMin(owner + slot, k);
      vslot[k] = (int)slot;
      return;
    }
    slot = (slot + 1) & mask;
  }
  atomicExch(status, (int)kBadIndex);  // table full (cannot happen at load <= 1/2)
  vslot[k] = 0;
}

// COMPON, step 2: a corner whose coordinates differ from its slot owner's is a hash collision
__global__ void k_vertex_check(int n, const double* __restrict__ geo, const int* __restrict__ owner,
                               const int* __restrict__ vslot, int* __restrict__ collide) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * n) return;
  const int o = owner[vslot[k]];
  double x, y, z, ox, oy, oz;
  corner(geo, k, x, y, z);
  corner(geo, o, ox, oy, oz);
  if (!(x == ox && y == oy && z == oz)) atomicExch(collide, 1);
}

__device__ __forceinline__ int find_root(const int* parent, int t) {
  // parents always point to smaller indices, so the walk ends
  while (true) {
    const int p = ((volatile const int*)parent)[t];
    if (p == t) return t;
    t = p;
  }
}

// COMPON, step 3 (one block): union-find over triangles joined through each vertex's first corner
// (hooking the larger root under the smaller, then path compression, until nothing changes); the
// root of a surface is its smallest triangle, so numbering the roots in order gives the surfaces
// in the order of their first triangles.  icomp = 1-based surface; out[0] = number of surfaces.
__global__ void __launch_bounds__(1024) k_components(int n, const int* __restrict__ owner,
                                                     const int* __restrict__ vslot, int* __restrict__ parent,
                                                     int* __restrict__ icomp, int* __restrict__ out, int* status) {
  __shared__ int s_changed, s_carry;
  __shared__ int s_scan[1024];
  for (int t = threadIdx.x; t < n; t += blockDim.x) parent[t] = t;
  __syncthreads();
  for (int it = 0;; ++it) {
    if (threadIdx.x == 0) s_changed = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < 3 * n; k += blockDim.x) {
      const int a = find_root(parent, k / 3), b = find_root(parent, owner[vslot[k]] / 3);
      if (a != b) {
        atomicMin(parent + max(a, b), min(a, b));
        s_changed = 1;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) parent[t] = find_root(parent, t);
    __syncthreads();
    if (!s_changed) break;
    if (it > 4 * 32) {  // far beyond the log-depth this needs
      if (threadIdx.x == 0) atomicExch(status, (int)kWaitTimeout);
      return;
    }
  }
  // number the roots in triangle order (block-wide exclusive scan in chunks of 1024)
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int b = 0; b < n; b += 1024) {
    const int t = b + threadIdx.x;
    const int f = (t < n && parent[t] == t) ? 1 : 0;
    s_scan[threadIdx.x] = f;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const int v = threadIdx.x >= off ? s_scan[threadIdx.x - off] : 0;
      __syncthreads();
      s_scan[threadIdx.x] += v;
      __syncthreads();
    }
    if (f) icomp[t] = s_carry + s_scan[threadIdx.x];  // 1-based label of the root
    __syncthreads();
    if (threadIdx.x == 1023) s_carry += s_scan[1023];
    __syncthreads();
  }
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int r = parent[t];
    if (r != t) icomp[t] = icomp[r];
  }
  // (roots were labelled before the loop above reads them: labels of roots are written in the
  // scan, and every non-root's parent is a root after compression)
  if (threadIdx.x == 0) out[0] = s_carry;
}

// COMPON, step 4: every edge (pair of vertex slots, ordered) counted in the edge table
__global__ void k_edge_insert(int n, const int* __restrict__ vslot, unsigned long long* __restrict__ keys,
                              int* __restrict__ count, unsigned mask, int* status) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * n) return;
  const int t = e / 3, c = e % 3;
  const unsigned a = (unsigned)vslot[3 * t + c], b = (unsigned)vslot[3 * t + (c + 1) % 3];
  const unsigned long long key = ((unsigned long long)min(a, b) << 32) | max(a, b);
  unsigned slot = (unsigned)mix64(key) & mask;
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const unsigned long long prev = atomicCAS(keys + slot, kEmpty, key);
    if (prev == kEmpty || prev == key) {
      atomicAdd(count + slot, 1);
      return;
    }
    slot = (slot + 1) & mask;
  }
  atomicExch(status, (int)kBadIndex);
}

// COMPON, step 5: open edges, and best.f:323-337: NDEF (1 with open edges, else the number of
// surfaces); with open edges every triangle is on surface 1.  out: [0] surfaces, [1] open edges,
// [2] NDEF.
__global__ void k_edge_open(const int* __restrict__ count, unsigned size, int* out) {
  int open = 0;
  for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < size; s += gridDim.x * blockDim.x) {
    const int c = count[s];
    open += (c != 0 && c != 2) ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) open += __shfl_xor_sync(0xffffffffu, open, o);
  if ((threadIdx.x & 31) == 0 && open) atomicAdd(out + 1, open);
}

__global__ void k_ndef(int n, int* __restrict__ icomp, int* __restrict__ out) {
  const int open = out[1], ncomp = out[0];
  const int ndef = (open > 0) ? 1 : (ncomp > 1 ? ncomp : 1);
  if (blockIdx.x == 0 && threadIdx.x == 0) out[2] = ndef;
  if (open > 0)
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) icomp[t] = 1;
}

// best.f:384-397: XMU = area * unit normal, per triangle
__global__ void k_xmu(int n, const double* __restrict__ geo, double* __restrict__ xmu) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double* p = geo + (size_t)t * kGeoStride;
  const double v21x = p[3] - p[0], v21y = p[4] - p[1], v21z = p[5] - p[2];
  const double v31x = p[6] - p[0], v31y = p[7] - p[1], v31z = p[8] - p[2];
  const double xnx = v31y * v21z - v31z * v21y, xny = v31z * v21x - v31x * v21z, xnz = v31x * v21y - v31y * v21x;
  const double xnl = sqrt(xnx * xnx + xny * xny + xnz * xnz);
  const double a = p[9];
  xmu[3 * (size_t)t] = a * xnx / xnl;
  xmu[3 * (size_t)t + 1] = a * xny / xnl;
  xmu[3 * (size_t)t + 2] = a * xnz / xnl;
}

// best.f:398-404 (NDEF = 1) and DEFGAM (NDEF > 1): GDEF = DIAGM / sum |XMU|^2, the sums in
// triangle order by one thread (the squares formed by the block)
__global__ void k_gdef(int n, int ndef, const double* __restrict__ xmu, const int* __restrict__ icomp,
                       const double* __restrict__ diagm, double* __restrict__ gdef) {
  __shared__ double sq[3][256];
  __shared__ int sk[256];
  const int nd = max(ndef, 1);
  double acc = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < nd; ++k) gdef[k] = 0.0;
  for (int b = 0; b < n; b += 256) {
    const int t = b + threadIdx.x;
    if (t < n) {
      const double x = xmu[3 * (size_t)t], y = xmu[3 * (size_t)t + 1], z = xmu[3 * (size_t)t + 2];
      sq[0][threadIdx.x] = x * x;
      sq[1][threadIdx.x] = y * y;
      sq[2][threadIdx.x] = z * z;
      sk[threadIdx.x] = ndef > 1 ? icomp[t] - 1 : 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int m = min(256, n - b);
      if (ndef <= 1) {
        for (int i = 0; i < m; ++i) acc = acc + sq[0][i] + sq[1][i] + sq[2][i];
      } else {
        for (int i = 0; i < m; ++i) gdef[sk[i]] = gdef[sk[i]] + sq[0][i] + sq[1][i] + sq[2][i];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double dm = *diagm;
    if (ndef <= 1) {
      gdef[0] = dm / acc;
    } else {
      for (int k = 0; k < ndef; ++k) gdef[k] = dm / gdef[k];
    }
  }
}

unsigned table_size(int n) {
  unsigned s = 1024;
  while (s < 6u * (unsigned)n) s <<= 1;
  return s;
}

}  // namespace

size_t setup_scratch_bytes(int n) {
  const size_t T = table_size(n);
  return T * (8 + 4) + T * (8 + 4) + (size_t)3 * n * 4 + (size_t)n * 4 + 256;
}

cudaError_t setup_device(int n, const double* tri, int iarea, double truearea, const SetupOut& o, void* scratch,
                         int* status, cudaStream_t s) {
  if (n <= 0) return cudaErrorInvalidValue;
  const unsigned T = table_size(n), mask = T - 1;
  unsigned char* p = static_cast<unsigned char*>(scratch);
  unsigned long long* vkeys = reinterpret_cast<unsigned long long*>(p);
  unsigned long long* ekeys = vkeys + T;
  int* owner = reinterpret_cast<int*>(ekeys + T);
  int* ecount = owner + T;
  int* vslot = ecount + T;
  int* parent = vslot + 3 * (size_t)n;
  int* flags = parent + n;  // [0] collision
  const int b3 = (3 * n + 255) / 256, b1 = (n + 255) / 256;
  cudaError_t e;
  k_centroid<<<1, 256, 0, s>>>(n, tri, o.scal + 2);
  BGPU_COUNT_LAUNCH();
  k_center_area<<<b1, 256, 0, s>>>(n, tri, o.scal + 2, o.geo, o.v, o.area);
  BGPU_COUNT_LAUNCH();
  k_area_total<<<1, 1024, 0, s>>>(n, iarea, truearea, o.area, o.geo, o.scal);
  BGPU_COUNT_LAUNCH();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // vertex table; rebuilt with another seed if two coordinate triples collide in the hash
  int collide = 1;
  unsigned long long seed = 0x243F6A8885A308D3ull;
  for (int attempt = 0; collide; ++attempt, seed = seed * 6364136223846793005ull + 1442695040888963407ull) {
    if (attempt == 8) return cudaErrorUnknown;  // eight 64-bit hash collisions in a row: not a real input
    if ((e = cudaMemsetAsync(vkeys, 0xFF, (size_t)T * 8, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(owner, 0x7F, (size_t)T * 4, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(flags, 0, 16, s)) != cudaSuccess) return e;
    k_vertex_insert<<<b3, 256, 0, s>>>(n, o.geo, seed, vkeys, owner, vslot, mask, status);
    BGPU_COUNT_LAUNCH();
    k_vertex_check<<<b3, 256, 0, s>>>(n, o.geo, owner, vslot, flags);
    BGPU_COUNT_LAUNCH();
    if ((e = cudaMemcpyAsync(&collide, flags, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  }
  if ((e = cudaMemsetAsync(o.counts, 0, 4 * sizeof(int), s)) != cudaSuccess) return e;
  k_components<<<1, 1024, 0, s>>>(n, owner, vslot, parent, o.icomp, o.counts, status);
  BGPU_COUNT_LAUNCH();
  if ((e = cudaMemsetAsync(ekeys, 0xFF, (size_t)T * 8, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(ecount, 0, (size_t)T * 4, s)) != cudaSuccess) return e;
  k_edge_insert<<<b3, 256, 0, s>>>(n, vslot, ekeys, ecount, mask, status);
  BGPU_COUNT_LAUNCH();
  k_edge_open<<<(T + 255) / 256 < 1184 ? (T + 255) / 256 : 1184, 256, 0, s>>>(ecount, T, o.counts);
  BGPU_COUNT_LAUNCH();
  k_ndef<<<b1, 256, 0, s>>>(n, o.icomp, o.counts);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t deflation_device(int n, int ndef, const double* geo, const int* icomp, const double* diagm, double* xmu,
                             double* gdef, cudaStream_t s) {
  if (n <= 0) return cudaErrorInvalidValue;
  k_xmu<<<(n + 255) / 256, 256, 0, s>>>(n, geo, xmu);
  BGPU_COUNT_LAUNCH();
  k_gdef<<<1, 256, 0, s>>>(n, ndef, xmu, icomp, diagm, gdef);
  BGPU_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace bgpu
