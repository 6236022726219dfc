// libbestgpu: BEST's solver seam (include/best_hmatrix.h) and its extensions (include/best_gpu.h)
// on one B200.
//
// Conventions kept from the reference's C interface (hmatrix/src/api.cpp): one solver per process
// in a global (api.cpp:127), messages queued and pulled one at a time (api.cpp:57-67, :881-890),
// every entry point guarded so that no exception crosses into Fortran and a failure is a nonzero
// status after a message (api.cpp:341-351), non-finite solutions reported as errors
// (api.cpp:681-689).  There is no CPU path: without a usable GPU, bhm_available() is 0 and every
// other call fails with a message.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <exception>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/best_driver.h"
#include "../../include/best_gpu.h"
#include "../../include/best_hmatrix.h"
#include "bgpu_internal.h"
#include "hmatrix.h"
#include "mixed.h"

namespace bgpu {

bool mesh_fast_ok(const double* v, long count, long stride_point, long stride_axis) {
  double side = 0.0;
  for (int a = 0; a < 3; ++a) {
    double lo = INFINITY, hi = -INFINITY;
    for (long p = 0; p < count; ++p) {
      const double x = v[a * stride_axis + p * stride_point];
      lo = std::min(lo, x);
      hi = std::max(hi, x);
    }
    side = std::max(side, hi - lo);
  }
  return std::isfinite(side) && side >= 1e-20 && side <= 1e20;
}

namespace {

// Messages for the caller's log (BEST appends them to its .log, best/besolve.f90:281-292): the
// library posts them, bhm_log_line hands them out oldest first, one per call.
class MessageQueue {
 public:
  void post(std::string m) { q_.push_back(std::move(m)); }
  // The oldest message, cut to `cap` bytes and without a terminator, removed from the queue; -1 when
  // the queue is empty.
  int take(char* out, int cap) {
    if (q_.empty()) return -1;
    std::string m = std::move(q_.front());
    q_.pop_front();
    const size_t len = std::min(m.size(), (size_t)std::max(cap, 0));
    if (len > 0) std::memcpy(out, m.data(), len);
    return (int)len;
  }

 private:
  std::deque<std::string> q_;
};
MessageQueue g_messages;

// Posts a printf-style message.
void note(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
void note(const char* fmt, ...) {
  va_list ap, ap2;
  va_start(ap, fmt);
  va_copy(ap2, ap);
  const int len = std::vsnprintf(nullptr, 0, fmt, ap);
  va_end(ap);
  std::string m(len > 0 ? (size_t)len : 0, '\0');
  if (len > 0) std::vsnprintf(&m[0], m.size() + 1, fmt, ap2);
  va_end(ap2);
  g_messages.post(std::move(m));
}

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// The exception boundary of every entry point: the body's status, or 1 with the reason posted when
// it throws, so that no C++ exception reaches the Fortran caller.
template <class Body>
int status_of(Body&& body) {
  std::string why;
  try {
    return body();
  } catch (const std::bad_alloc&) {
    why = "host memory exhausted";
  } catch (const std::exception& e) {
    why = e.what();
  } catch (...) {
    why = "unexpected failure";
  }
  note("error: %s", why.c_str());
  return 1;
}

// Device buffer that frees itself.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // (Re)allocates when smaller than `need`; zeroes fresh memory when `zero`.
  void ensure(size_t need, const char* what, bool zero = false) {
    if (bytes >= need && p) return;
    reset();
    cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
      size_t fr = 0, tot = 0;
      cudaGetLastError();
      cudaMemGetInfo(&fr, &tot);
      throw CudaError(std::string("cannot allocate ") + what + ": " + std::to_string(need / 1e9) +
                      " GB needed, " + std::to_string(fr / 1e9) + " GB free on the GPU");
    }
    bytes = need;
    if (zero) ck(cudaMemset(p, 0, need), "cudaMemset");
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

long padded_ld(int n) { return ((long)n + 31) / 32 * 32; }

struct Runtime {
  int device = -1;
  cudaStream_t stream = nullptr;
  DevBuf status, info;     // device status word, dgetrf info
  DevBuf lu_scratch;       // grid-barrier words and pivot candidates
  DevBuf trsv_scratch;     // flags, ticket and the permuted right-hand sides
  cudaEvent_t ev[8] = {};
  double ms[8] = {};
  Runtime() {
    int count = 0;
    if (cudaGetDevice(&device) != cudaSuccess || cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw CudaError("no CUDA device is usable");
    }
    ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
    status.ensure(256, "status words", true);
    info.ensure(256, "info", true);
    lu_scratch.ensure(lu_scratch_bytes(0), "LU scratch", true);
  }
  ~Runtime() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
  void sync(const char* what) { ck(cudaStreamSynchronize(stream), what); }
  // Reads and clears the device status word; throws on a recorded failure.
  void check_status(const char* what) {
    int st = 0;
    ck(cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, stream), "status read");
    sync(what);
    if (st != kOk) {
      ck(cudaMemsetAsync(status.p, 0, sizeof(int), stream), "status clear");
      sync(what);
      if (st == kWaitTimeout)
        throw CudaError(std::string(what) + ": a device-side wait ran out (kernel gave up, no result)");
      if (st == kNotFinite) throw CudaError(std::string(what) + ": the solution is not finite (NaN or Inf)");
      throw CudaError(std::string(what) + ": device status " + std::to_string(st));
    }
  }
  void ensure_trsv(int n) { trsv_scratch.ensure(trsv_scratch_bytes(n), "solve scratch", true); }
  float elapsed(int a, int b) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, ev[a], ev[b]) != cudaSuccess) {
      cudaGetLastError();
      t = 0.f;
    }
    return t;
  }
};

std::unique_ptr<Runtime> g_rt;

Runtime& rt() {
  if (!g_rt) g_rt = std::make_unique<Runtime>();
  return *g_rt;
}

struct Solver {
  int n = 0;
  double afac = 1.0, cg = 1.0;
  std::vector<double> x_host;  // incenters, n x 3 column-major
  std::vector<double> v_host[3], area_host;  // the mesh as given (corners, corrected areas)
  int ndef = 0;                               // deflation of the last build (host copies)
  std::vector<double> gdef_host, xmu_host;
  std::vector<int> comp_host;
  DevBuf geo, xc, self9, diag;
  DevBuf gr;                   // GR / its LU factors (FP64), n x ld
  long ld = 0;
  DevBuf ipiv, perm, dl64, du64;  // pivots, composed permutation, diagonal-block inverses
  DevBuf gdef, comp, xmu;
  DevBuf rhs, rhs_keep;        // right-hand sides (host-interface staging, and a kept copy)
  // set up on the device (bgpu_create_from_triangles): the triangles as read, BEST's V1/V2/V3 and
  // areas, {AFAC, total area, centroid}, {surfaces, open edges, NDEF}, scratch of the hash tables
  bool prepared = false;
  int counts_host[3] = {0, 0, 0};
  double scal_host[5] = {0, 0, 0, 0, 0};
  DevBuf tri, vset, area, scal, counts, setup_scratch;
  std::unique_ptr<MixedSolver> mixed;
  std::unique_ptr<HMatrixSolver> hmat;  // the H-matrix path (BGPU_HMATRIX)
  int precision = BGPU_FP64;
  bool factored = false;
  bool fast_ok = true;  // mesh_fast_ok of the mesh
  DevMesh mesh() const {
    DevMesh m;
    m.n = n;
    m.cg = cg;
    m.afac = afac;
    m.fast_ok = fast_ok;
    m.geo = geo.as<double>();
    m.xc = xc.as<double>();
    m.self9 = self9.as<double>();
    return m;
  }
};

std::unique_ptr<Solver> g;
int g_prec_override = -1;
int g_refine[2] = {8, 10};  // GMRES restarts, Krylov vectors per restart
double g_solve_info[2] = {0, 0};  // refinement iterations, relative residual of the last solve
struct HOpts {
  int leaf = 128;
  double eta = 2.0;
  int kmax = 90;
} g_hm_opts;  // H-matrix settings (bgpu_hmatrix_set_options)

Solver& solver() {
  if (!g) throw std::runtime_error("bhm_create has not been called");
  return *g;
}

int precision_for(int direct, int single) {
  if (g_prec_override >= 0) return g_prec_override;
  if (const char* e = std::getenv("BEST_GPU_PRECISION")) {
    if (!std::strcmp(e, "fp64")) return BGPU_FP64;
    if (!std::strcmp(e, "mixed")) return BGPU_MIXED;
    if (!std::strcmp(e, "hmatrix")) return BGPU_HMATRIX;
  }
  if (direct && !single) return BGPU_FP64;
  return BGPU_MIXED;
}

// Factors the FP64 matrix in s.gr (dgetrf); throws on a zero pivot.
void factor64(Solver& s, Runtime& r) {
  const int n3 = 3 * s.n;
  s.ipiv.ensure(sizeof(int) * n3, "pivots");
  s.perm.ensure(sizeof(int) * n3, "permutation");
  LuScratch ws{r.lu_scratch.p, r.lu_scratch.bytes};
  ck(lu64_getrf(s.gr.as<double>(), s.ld, n3, s.ipiv.as<int>(), r.info.as<int>(), r.status.as<int>(), ws, r.stream),
     "LU");
  ck(lu_perm_from_ipiv(s.ipiv.as<int>(), n3, s.perm.as<int>(), r.stream), "permutation");
  s.dl64.ensure(diag_inverse_elems(n3) * sizeof(double), "diagonal-block inverses (L)");
  s.du64.ensure(diag_inverse_elems(n3) * sizeof(double), "diagonal-block inverses (U)");
  ck(diag_inverses64(s.gr.as<double>(), s.ld, n3, s.dl64.as<double>(), s.du64.as<double>(), r.stream),
     "diagonal inverses");
}

void solve_device(Solver& s, Runtime& r, int nrhs, double* d_b, long ldb) {
  if (!s.factored) throw std::runtime_error("bhm_build has not factored GR");
  const int n3 = 3 * s.n;
  ck(cudaEventRecord(r.ev[6], r.stream), "event");
  if (s.precision == BGPU_HMATRIX && s.hmat) {
    HReport rep{};
    try {
      s.hmat->solve(nrhs, d_b, ldb, r.stream, &rep);
    } catch (const std::runtime_error& e) {
      throw CudaError(e.what());
    }
    g_solve_info[0] = rep.iterations;
    g_solve_info[1] = rep.relres;
  } else if (s.precision == BGPU_MIXED && s.mixed) {
    MixedReport rep{};
    // keep the right-hand sides: a failed refinement falls back to the FP64 LU on the same input
    s.rhs_keep.ensure((size_t)n3 * nrhs * sizeof(double), "right-hand sides (copy)");
    ck(cudaMemcpy2DAsync(s.rhs_keep.p, (size_t)n3 * sizeof(double), d_b, (size_t)ldb * sizeof(double),
                         (size_t)n3 * sizeof(double), nrhs, cudaMemcpyDeviceToDevice, r.stream),
       "rhs copy");
    try {
      s.mixed->solve(nrhs, d_b, ldb, r.stream, &rep);
      g_solve_info[0] = rep.iterations;
      g_solve_info[1] = rep.relres;
    } catch (const MixedFailure& e) {
      note("mixed precision: %s; factoring the FP64 matrix instead", e.what());
      ck(cudaMemcpy2DAsync(d_b, (size_t)ldb * sizeof(double), s.rhs_keep.p, (size_t)n3 * sizeof(double),
                           (size_t)n3 * sizeof(double), nrhs, cudaMemcpyDeviceToDevice, r.stream),
         "rhs restore");
      factor64(s, r);
      r.check_status("FP64 fallback");
      s.precision = BGPU_FP64;
      solve_device(s, r, nrhs, d_b, ldb);
      return;
    }
  } else {
    r.ensure_trsv(n3);
    for (int c = 0; c < nrhs; c += 16) {
      const int q = std::min(16, nrhs - c);
      ck(getrs64_inv(s.gr.as<double>(), s.ld, s.dl64.as<double>(), s.du64.as<double>(), n3, s.perm.as<int>(),
                     d_b + (size_t)c * ldb, ldb, q, r.trsv_scratch.p, r.status.as<int>(), r.stream),
         "solve");
    }
    g_solve_info[0] = 0;
    g_solve_info[1] = 0;
  }
  ck(check_finite(d_b, ldb, n3, nrhs, r.status.as<int>(), r.stream), "finite check");
  ck(cudaEventRecord(r.ev[7], r.stream), "event");
  r.check_status("solve");
  r.ms[3] = r.elapsed(6, 7);
}

// host mesh arrays (v1, v2, v3: n x 3 column-major; area) in the device layout, kGeoStride per triangle
std::vector<double> geo_host(int n, const double* v1, const double* v2, const double* v3, const double* area) {
  std::vector<double> h((size_t)n * kGeoStride, 0.0);
  for (int t = 0; t < n; ++t) {
    for (int c = 0; c < 3; ++c) {
      h[(size_t)t * kGeoStride + c] = v1[(size_t)c * n + t];
      h[(size_t)t * kGeoStride + 3 + c] = v2[(size_t)c * n + t];
      h[(size_t)t * kGeoStride + 6 + c] = v3[(size_t)c * n + t];
    }
    h[(size_t)t * kGeoStride + 9] = area[t];
  }
  return h;
}

// A series of meshes of one body (BEST's workflow of results extrapolated in 1/N, best/best.f:154-157),
// assembled, factored (FP64, partial pivoting) and solved together.  Mesh i's arrays sit in
// concatenated buffers from triangle t0[i]; its GR (order 3 n_i, leading dimension ld[i]) from gr0[i].
struct Series {
  int count = 0;
  double cg = 1.0;
  std::vector<int> n;
  std::vector<long> t0;        // first triangle of each mesh
  std::vector<double> afac;
  std::vector<double> x_host;  // incenters: mesh i's n_i x 3 column-major block at 3 t0[i]
  DevBuf geo, xc, self9, diag;
  std::vector<int> ndef;
  std::vector<long> gdef0;     // first deflation weight of each mesh
  DevBuf gdef, comp, xmu;
  std::vector<long> ld;
  std::vector<size_t> gr0, inv0;
  DevBuf gr, ipiv, perm, dl, du, info, rhs;
  cudaGraphExec_t graph = nullptr;  // assembly + LU + permutations + diagonal inverses of the series
  unsigned long long graph_kernels = 0;
  bool graph_tried = false, factored = false;
  double ms[4] = {};  // build (graph), of which assembly; last solve; tuning pass
  // BGPU_MIXED (bgpu_series_set_precision): each mesh's BF16 tensor-core factorisation on a stream
  // of its own, all enqueued before any is waited for; FP64 GMRES-IR solves
  int precision = BGPU_FP64;
  int built_precision = BGPU_FP64;
  std::vector<std::unique_ptr<MixedSolver>> mixed;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> ev_done;
  ~Series() {
    if (graph) cudaGraphExecDestroy(graph);
    for (cudaStream_t q : streams) cudaStreamDestroy(q);
    for (cudaEvent_t e : ev_done) cudaEventDestroy(e);
  }
  std::vector<char> fast_ok;  // mesh_fast_ok of each mesh
  DevMesh mesh(int i) const {
    DevMesh m;
    m.n = n[i];
    m.cg = cg;
    m.afac = afac[i];
    m.fast_ok = fast_ok[i] != 0;
    m.geo = geo.as<double>() + (size_t)t0[i] * kGeoStride;
    m.xc = xc.as<double>() + (size_t)t0[i] * kXcStride;
    m.self9 = self9.as<double>() + (size_t)t0[i] * 9;
    return m;
  }
  long rows() const { return 3 * (t0[count - 1] + n[count - 1]); }
};

std::unique_ptr<Series> g_series;

Series& series() {
  if (!g_series) throw std::runtime_error("bgpu_series_create has not been called");
  return *g_series;
}

// every device step of a series build, on stream st (run directly, or captured into the graph);
// ev_assembled (direct runs only) is recorded after the assembly
void series_record(Series& S, Runtime& r, cudaStream_t st, cudaEvent_t ev_assembled = nullptr) {
  SeriesAssembly sa;
  sa.count = S.count;
  for (int i = 0; i < S.count; ++i) {
    sa.mesh[i] = S.mesh(i);
    DevDeflation d;
    if (S.ndef[i] >= 1) {
      d.ndef = S.ndef[i];
      d.gdef = S.gdef.as<double>() + S.gdef0[i];
      d.xmu = S.xmu.as<double>() + 3 * S.t0[i];
      if (S.ndef[i] > 1) d.comp = S.comp.as<int>() + S.t0[i];
    }
    sa.defl[i] = d;
    sa.out[i] = S.gr.as<double>() + S.gr0[i];
    sa.ld[i] = S.ld[i];
  }
  ck(launch_assemble_series(sa, st), "series assembly");
  if (ev_assembled) ck(cudaEventRecord(ev_assembled, st), "event");
  std::vector<LuItem> items(S.count);
  for (int i = 0; i < S.count; ++i)
    items[i] = LuItem{S.gr.as<double>() + S.gr0[i], S.ld[i], 3 * S.n[i], S.ipiv.as<int>() + 3 * S.t0[i],
                      S.info.as<int>() + i};
  LuScratch ws{r.lu_scratch.p, r.lu_scratch.bytes};
  ck(lu64_getrf_batch(items.data(), S.count, r.status.as<int>(), ws, st), "series LU");
  for (int i = 0; i < S.count; ++i) {
    const int n3 = 3 * S.n[i];
    ck(lu_perm_from_ipiv(S.ipiv.as<int>() + 3 * S.t0[i], n3, S.perm.as<int>() + 3 * S.t0[i], st), "permutation");
    ck(diag_inverses64(S.gr.as<double>() + S.gr0[i], S.ld[i], n3, S.dl.as<double>() + S.inv0[i],
                       S.du.as<double>() + S.inv0[i], st),
       "diagonal inverses");
  }
}

// The mixed-precision series build: every mesh's assembly and BF16 tensor-core factorisation
// enqueued on its own stream (after the deflation uploads on the runtime stream), then all waited
// for.  Throws MixedFailure when a mesh cannot be factored without pivoting.
void series_build_mixed(Series& S, Runtime& r) {
  if ((int)S.mixed.size() != S.count) {
    S.mixed.clear();
    for (int i = 0; i < S.count; ++i) S.mixed.push_back(std::make_unique<MixedSolver>());
  }
  while ((int)S.streams.size() < S.count) {
    cudaStream_t q;
    cudaEvent_t e;
    ck(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking), "series stream");
    ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "series event");
    S.streams.push_back(q);
    S.ev_done.push_back(e);
  }
  ck(cudaEventRecord(r.ev[2], r.stream), "event");
  for (int i = 0; i < S.count; ++i) {
    DevDeflation d;
    if (S.ndef[i] >= 1) {
      d.ndef = S.ndef[i];
      d.gdef = S.gdef.as<double>() + S.gdef0[i];
      d.xmu = S.xmu.as<double>() + 3 * S.t0[i];
      if (S.ndef[i] > 1) d.comp = S.comp.as<int>() + S.t0[i];
    }
    ck(cudaStreamWaitEvent(S.streams[i], r.ev[2], 0), "series fork");
    S.mixed[i]->set_refinement(g_refine[0], g_refine[1]);
    S.mixed[i]->build(S.mesh(i), d, S.gr.as<double>() + S.gr0[i], S.ld[i], 1e-10, S.streams[i], S.ev_done[i],
                      S.ev_done[i], false);
  }
  for (int i = 0; i < S.count; ++i) {
    S.mixed[i]->finish_build(S.streams[i]);
    ck(cudaStreamWaitEvent(r.stream, S.ev_done[i], 0), "series join");
  }
  ck(cudaEventRecord(r.ev[4], r.stream), "event");
}

// Assembly (with the deflation defl, on the device), factorisation and the host-side report: the
// part of bhm_build after the deflation vectors are in place.
int build_common(Solver& s, Runtime& r, double eps, int direct, int single, const DevDeflation& defl) {
  const int n = s.n, n3 = 3 * n;
  s.factored = false;
  s.precision = precision_for(direct, single);
  if (s.precision != BGPU_HMATRIX) {
    // the dense paths hold the FP64 GR (72 N^2 bytes; the mixed path an FP32 copy beside it):
    // beyond the free device memory, the H-matrix path takes over (as the reference switches to
    // its H-matrix for large N, best/best.f:138)
    size_t fr = 0, tot = 0;
    ck(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
    // memory this solver holds now is reused or freed by the build: count it as available
    const double held = (double)s.gr.bytes + (s.mixed ? (double)s.mixed->device_bytes() : 0.0);
    const double need = (s.precision == BGPU_FP64 ? 72.0 : 108.0) * (double)n * n * 1.02 + 5.12e8 - held;
    if (need > (double)fr) {
      note("dense GR of order %d needs %.1f GB, %.1f GB free on the GPU: H-matrix path", n3, need / 1e9, fr / 1e9);
      s.precision = BGPU_HMATRIX;
    }
  }
  if (s.precision == BGPU_HMATRIX) {
    s.gr.reset();
    s.mixed.reset();
    if (!s.hmat) s.hmat = std::make_unique<HMatrixSolver>();
    s.hmat->set_options(g_hm_opts.leaf, g_hm_opts.eta, g_hm_opts.kmax);
    ck(cudaEventRecord(r.ev[2], r.stream), "event");
    try {
      s.hmat->build(s.mesh(), defl, defl.ndef, eps, r.stream);
    } catch (const std::runtime_error& e) {
      throw CudaError(e.what());
    }
    ck(cudaEventRecord(r.ev[5], r.stream), "event");
    r.sync("bhm_build");
    const std::vector<double> st = s.hmat->stats();
    r.ms[1] = st[9] + st[10];
    r.ms[2] = st[11];
    r.ms[4] = r.elapsed(2, 5);
    s.factored = true;
    note("GPU build: H-matrix of order %d at eps %.0e: %d leaves, %d dense blocks (%.2f GB), %d low-rank blocks "
         "(%.2f GB, mean rank %.1f, largest %d, %d at the cap), fill %.1f ms, cross approximation %.1f ms, "
         "block-Jacobi preconditioner %.1f ms",
         n3, eps, (int)st[1], (int)st[2], st[4] * 8e-9, (int)st[3], st[5] * 8e-9, st[6], (int)st[7], (int)st[8], st[9],
         st[10], st[11]);
    return 0;
  }
  s.hmat.reset();
  s.ld = padded_ld(n3);
  s.gr.ensure((size_t)s.ld * n3 * sizeof(double), "GR (FP64)");
  ck(cudaEventRecord(r.ev[2], r.stream), "event");
  if (s.precision == BGPU_MIXED) {
    if (!s.mixed) s.mixed = std::make_unique<MixedSolver>();
    s.mixed->set_refinement(g_refine[0], g_refine[1]);
    try {
      s.mixed->build(s.mesh(), defl, s.gr.as<double>(), s.ld, eps, r.stream, r.ev[3], r.ev[4]);
    } catch (const MixedFailure& e) {
      note("mixed precision: %s; factoring the FP64 matrix instead", e.what());
      s.precision = BGPU_FP64;
      factor64(s, r);
    }
    ck(cudaEventRecord(r.ev[5], r.stream), "event");
    r.check_status("bhm_build");
  } else {
    ck(launch_assemble(s.mesh(), 0, n, 0, n, s.gr.as<double>(), s.ld, defl, nullptr, 0, r.stream), "assembly");
    ck(cudaEventRecord(r.ev[3], r.stream), "event");
    factor64(s, r);
    ck(cudaEventRecord(r.ev[5], r.stream), "event");
    ck(cudaEventRecord(r.ev[4], r.stream), "event");
    r.check_status("bhm_build");
    ck(cudaEventRecord(r.ev[4], r.stream), "event");
  }
  r.sync("bhm_build");
  int info = 0;
  ck(cudaMemcpy(&info, r.info.p, sizeof(int), cudaMemcpyDeviceToHost), "info read");
  r.ms[1] = r.elapsed(2, 3);
  r.ms[2] = r.elapsed(3, 5);
  r.ms[4] = r.elapsed(2, 5);
  if (info > 0) {
    note("error: the LU factorisation found U(%d,%d) = 0: GR is singular", info, info);
    return 1;
  }
  s.factored = true;
  if (s.mixed)
    for (auto& line : s.mixed->profile_report()) note("%s", line.c_str());
  note("GPU build: %s LU of order %d, assembly %.1f ms, factorisation %.1f ms (%.1f TFLOP/s)",
       s.precision == BGPU_FP64 ? "FP64" : (s.mixed ? s.mixed->name() : "mixed"), n3, r.ms[1], r.ms[2],
       (2.0 / 3.0) * (double)n3 * n3 * n3 / (r.ms[2] * 1e-3) / 1e12);
  return 0;
}

}  // namespace

void log_message(const char* msg) { g_messages.post(msg); }

}  // namespace bgpu

using namespace bgpu;

extern "C" {

int bhm_available(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return count > 0 ? 1 : 0;
}

int bhm_create(int n, const double* v1, const double* v2, const double* v3, const double* area, double afac,
               double cg, int /*threads*/) {
  return status_of([&] {
    if (n < 1) {
      note("error: the GPU solver needs at least 1 triangle");
      return 1;
    }
    Runtime& r = rt();
    auto s = std::make_unique<Solver>();
    s->n = n;
    s->afac = afac;
    s->cg = cg;
    std::vector<double> h = geo_host(n, v1, v2, v3, area);
    s->fast_ok = mesh_fast_ok(v1, n, 1, n) && mesh_fast_ok(v2, n, 1, n) && mesh_fast_ok(v3, n, 1, n);
    s->v_host[0].assign(v1, v1 + 3 * (size_t)n);
    s->v_host[1].assign(v2, v2 + 3 * (size_t)n);
    s->v_host[2].assign(v3, v3 + 3 * (size_t)n);
    s->area_host.assign(area, area + n);
    s->geo.ensure(h.size() * sizeof(double), "mesh");
    s->xc.ensure((size_t)n * kXcStride * sizeof(double), "incenters");
    s->self9.ensure((size_t)n * 9 * sizeof(double), "self blocks");
    s->diag.ensure(256, "diagonal mean");
    ck(cudaEventRecord(r.ev[0], r.stream), "event");
    ck(cudaMemcpyAsync(s->geo.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, r.stream), "mesh copy");
    ck(launch_self_blocks(s->mesh(), r.stream), "self blocks");
    std::vector<double> xc((size_t)n * kXcStride);
    ck(cudaMemcpyAsync(xc.data(), s->xc.p, xc.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream),
       "incenter copy");
    ck(cudaEventRecord(r.ev[1], r.stream), "event");
    r.sync("bhm_create");
    r.ms[0] = r.elapsed(0, 1);
    s->x_host.resize((size_t)3 * n);
    for (int t = 0; t < n; ++t)
      for (int c = 0; c < 3; ++c) s->x_host[(size_t)c * n + t] = xc[(size_t)t * kXcStride + c];
    g = std::move(s);
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, r.device);
    note("GPU solver: %d triangles on %s (%d SMs, %.0f GB), dense GR %.2f GB in FP64", n, prop.name,
        prop.multiProcessorCount, prop.totalGlobalMem / 1e9, 72.0 * n * (double)n / 1e9);
    return 0;
  });
}

int bgpu_create_from_triangles(int n, const double* tri, int iarea, double truearea, double cg, double* info,
                               int* counts) {
  return status_of([&] {
    if (n < 1) {
      note("error: the GPU solver needs at least 1 triangle");
      return 1;
    }
    Runtime& r = rt();
    auto s = std::make_unique<Solver>();
    s->n = n;
    s->cg = cg;
    s->prepared = true;
    s->fast_ok = mesh_fast_ok(tri, 3 * (long)n, 3, 1);
    s->tri.ensure((size_t)9 * n * sizeof(double), "triangles");
    s->geo.ensure((size_t)n * kGeoStride * sizeof(double), "mesh");
    s->vset.ensure((size_t)9 * n * sizeof(double), "centred corners");
    s->area.ensure((size_t)n * sizeof(double), "areas");
    s->scal.ensure(8 * sizeof(double), "set-up scalars");
    s->counts.ensure(4 * sizeof(int), "surface counts");
    s->comp.ensure((size_t)n * sizeof(int), "surface labels");
    s->setup_scratch.ensure(setup_scratch_bytes(n), "set-up hash tables");
    s->xc.ensure((size_t)n * kXcStride * sizeof(double), "incenters");
    s->self9.ensure((size_t)n * 9 * sizeof(double), "self blocks");
    s->diag.ensure(256, "diagonal mean");
    ck(cudaEventRecord(r.ev[0], r.stream), "event");
    ck(cudaMemcpyAsync(s->tri.p, tri, (size_t)9 * n * sizeof(double), cudaMemcpyHostToDevice, r.stream), "mesh copy");
    SetupOut o;
    o.geo = s->geo.as<double>();
    o.v = s->vset.as<double>();
    o.area = s->area.as<double>();
    o.scal = s->scal.as<double>();
    o.icomp = s->comp.as<int>();
    o.counts = s->counts.as<int>();
    ck(setup_device(n, s->tri.as<double>(), iarea, truearea, o, s->setup_scratch.p, r.status.as<int>(), r.stream),
       "set-up on the device");
    ck(cudaMemcpyAsync(s->scal_host, s->scal.p, 5 * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "set-up copy");
    ck(cudaMemcpyAsync(s->counts_host, s->counts.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, r.stream), "counts copy");
    r.sync("bgpu_create_from_triangles");
    s->afac = s->scal_host[0];  // the self blocks scale by sqrt(AFAC) (best/tgetgr.f:107-112)
    // what bhm_create does with a mesh given by the caller: self blocks, incenters, DIAGM
    ck(launch_self_blocks(s->mesh(), r.stream), "self blocks");
    ck(launch_diag_mean(s->mesh(), s->diag.as<double>(), r.stream), "diagonal mean");
    std::vector<double> xc((size_t)n * kXcStride), v((size_t)9 * n);
    s->area_host.resize(n);
    ck(cudaMemcpyAsync(xc.data(), s->xc.p, xc.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream),
       "incenter copy");
    ck(cudaMemcpyAsync(v.data(), s->vset.p, v.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "corner copy");
    ck(cudaMemcpyAsync(s->area_host.data(), s->area.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, r.stream),
       "area copy");
    ck(cudaEventRecord(r.ev[1], r.stream), "event");
    r.sync("bgpu_create_from_triangles");
    r.check_status("bgpu_create_from_triangles");
    r.ms[0] = r.elapsed(0, 1);
    for (int c = 0; c < 3; ++c) s->v_host[c].assign(v.begin() + (size_t)c * 3 * n, v.begin() + (size_t)(c + 1) * 3 * n);
    s->x_host.resize((size_t)3 * n);
    for (int t = 0; t < n; ++t)
      for (int c = 0; c < 3; ++c) s->x_host[(size_t)c * n + t] = xc[(size_t)t * kXcStride + c];
    if (info)
      for (int q = 0; q < 5; ++q) info[q] = s->scal_host[q];
    if (counts)
      for (int q = 0; q < 3; ++q) counts[q] = s->counts_host[q];
    note("GPU set-up: %d triangles, %d surface(s), %d open edge(s), NDEF %d, AFAC %.15g (%.2f ms on the device)", n,
         s->counts_host[0], s->counts_host[1], s->counts_host[2], s->afac, r.ms[0]);
    g = std::move(s);
    return 0;
  });
}

int bgpu_build_prepared(double eps, int direct, int single, int /*nrhs*/) {
  return status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    if (!s.prepared) {
      note("error: bgpu_build_prepared needs a mesh set up by bgpu_create_from_triangles");
      return 1;
    }
    const int n = s.n, n3 = 3 * n, ndef = s.counts_host[2];
    s.ndef = ndef;
    s.gdef.ensure(sizeof(double) * std::max(ndef, 1), "deflation weights");
    s.xmu.ensure(sizeof(double) * n3, "deflation vectors");
    ck(deflation_device(n, ndef, s.geo.as<double>(), s.comp.as<int>(), s.diag.as<double>(), s.xmu.as<double>(),
                        s.gdef.as<double>(), r.stream),
       "deflation on the device");
    s.gdef_host.resize(ndef);
    s.xmu_host.resize(n3);
    s.comp_host.resize(ndef > 1 ? n : 0);
    ck(cudaMemcpyAsync(s.gdef_host.data(), s.gdef.p, sizeof(double) * ndef, cudaMemcpyDeviceToHost, r.stream), "gdef");
    ck(cudaMemcpyAsync(s.xmu_host.data(), s.xmu.p, sizeof(double) * n3, cudaMemcpyDeviceToHost, r.stream), "xmu");
    if (ndef > 1)
      ck(cudaMemcpyAsync(s.comp_host.data(), s.comp.p, sizeof(int) * n, cudaMemcpyDeviceToHost, r.stream), "comp");
    DevDeflation defl;
    defl.ndef = ndef;
    defl.gdef = s.gdef.as<double>();
    defl.xmu = s.xmu.as<double>();
    defl.comp = ndef > 1 ? s.comp.as<int>() : nullptr;
    return build_common(s, r, eps, direct, single, defl);
  });
}

int bgpu_prepared_arrays(double* v1, double* v2, double* v3, double* area, int* icomp, double* xmu, double* gdef) {
  return status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    if (!s.prepared) {
      note("error: bgpu_prepared_arrays needs a mesh set up by bgpu_create_from_triangles");
      return 1;
    }
    const size_t n = (size_t)s.n;
    double* vs[3] = {v1, v2, v3};
    for (int c = 0; c < 3; ++c)
      if (vs[c]) std::memcpy(vs[c], s.v_host[c].data(), 3 * n * sizeof(double));
    if (area) std::memcpy(area, s.area_host.data(), n * sizeof(double));
    if (icomp) {
      ck(cudaMemcpyAsync(icomp, s.comp.p, n * sizeof(int), cudaMemcpyDeviceToHost, r.stream), "labels");
      r.sync("bgpu_prepared_arrays");
    }
    if (xmu && s.xmu_host.size() == 3 * n) std::memcpy(xmu, s.xmu_host.data(), 3 * n * sizeof(double));
    if (gdef) std::memcpy(gdef, s.gdef_host.data(), s.gdef_host.size() * sizeof(double));
    return 0;
  });
}

void bhm_incenters(double* x) {
  status_of([&] {
    Solver& s = solver();
    std::memcpy(x, s.x_host.data(), s.x_host.size() * sizeof(double));
    return 0;
  });
}

void bhm_entries(int i0, int m, int j0, int nc, double* a, int lda) {
  status_of([&] {
    if (m <= 0 || nc <= 0) return 0;
    Solver& s = solver();
    Runtime& r = rt();
    if (i0 < 0 || j0 < 0 || (long)i0 + m > 3L * s.n || (long)j0 + nc > 3L * s.n || lda < m) {
      note("error: bhm_entries: rows %d..%d or columns %d..%d outside GR (order %d), or lda %d < m", i0, i0 + m - 1, j0,
          j0 + nc - 1, 3 * s.n, lda);
      return 1;
    }
    const int t0 = i0 / 3, t1 = (i0 + m - 1) / 3 + 1;
    const long rows = 3L * (t1 - t0);
    // columns in chunks so the staging buffer stays below ~1 GB
    const int cmax = std::max(1, (int)std::min<long>((long)s.n, (1L << 27) / std::max(1L, rows) / 3));
    const int s0 = j0 / 3, s1 = (j0 + nc - 1) / 3 + 1;
    DevBuf tmp;
    tmp.ensure((size_t)rows * 3 * std::min(cmax, s1 - s0) * sizeof(double), "entry staging");
    for (int c = s0; c < s1; c += cmax) {
      const int ce = std::min(s1, c + cmax);
      DevDeflation none;
      ck(launch_assemble(s.mesh(), t0, t1, c, ce, tmp.as<double>(), rows, none, nullptr, 0, r.stream), "entries");
      // copy the part of columns [3c, 3ce) x rows [3 t0, 3 t1) that the caller asked for
      const int jlo = std::max(j0, 3 * c), jhi = std::min(j0 + nc, 3 * ce);
      const double* src = tmp.as<double>() + (size_t)(jlo - 3 * c) * rows + (i0 - 3 * t0);
      double* dst = a + (size_t)(jlo - j0) * lda;
      ck(cudaMemcpy2DAsync(dst, (size_t)lda * sizeof(double), src, (size_t)rows * sizeof(double),
                           (size_t)m * sizeof(double), (size_t)(jhi - jlo), cudaMemcpyDeviceToHost, r.stream),
         "entries copy");
      r.sync("bhm_entries");
    }
    return 0;
  });
}

double bhm_diag_mean(void) {
  double v = 0.0;
  status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    ck(launch_diag_mean(s.mesh(), s.diag.as<double>(), r.stream), "diagonal mean");
    ck(cudaMemcpyAsync(&v, s.diag.p, sizeof(double), cudaMemcpyDeviceToHost, r.stream), "diagonal copy");
    r.sync("bhm_diag_mean");
    return 0;
  });
  return v;
}

int bhm_build(double eps, int direct, double /*eps_pre*/, int ndef, const double* gdef, const int* comp,
              const double* xmu, int single, int /*nrhs*/) {
  return status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    const int n = s.n, n3 = 3 * n;
    DevDeflation defl;
    s.ndef = std::max(0, ndef);
    s.gdef_host.assign(gdef, gdef + s.ndef);
    s.xmu_host.assign(xmu, xmu + (ndef >= 1 ? n3 : 0));
    s.comp_host.assign(comp, comp + (ndef > 1 ? n : 0));
    if (ndef >= 1) {
      s.gdef.ensure(sizeof(double) * ndef, "deflation weights");
      s.xmu.ensure(sizeof(double) * n3, "deflation vectors");
      ck(cudaMemcpyAsync(s.gdef.p, gdef, sizeof(double) * ndef, cudaMemcpyHostToDevice, r.stream), "gdef copy");
      ck(cudaMemcpyAsync(s.xmu.p, xmu, sizeof(double) * n3, cudaMemcpyHostToDevice, r.stream), "xmu copy");
      defl.ndef = ndef;
      defl.gdef = s.gdef.as<double>();
      defl.xmu = s.xmu.as<double>();
      if (ndef > 1) {
        s.comp.ensure(sizeof(int) * n, "surface labels");
        ck(cudaMemcpyAsync(s.comp.p, comp, sizeof(int) * n, cudaMemcpyHostToDevice, r.stream), "comp copy");
        defl.comp = s.comp.as<int>();
      }
    }
    return build_common(s, r, eps, direct, single, defl);
  });
}

int bhm_solve(int nrhs, double* b) {
  return status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    if (nrhs <= 0) return 0;
    const int n3 = 3 * s.n;
    s.rhs.ensure((size_t)n3 * nrhs * sizeof(double), "right-hand sides");
    ck(cudaMemcpyAsync(s.rhs.p, b, (size_t)n3 * nrhs * sizeof(double), cudaMemcpyHostToDevice, r.stream), "b copy");
    solve_device(s, r, nrhs, s.rhs.as<double>(), n3);
    ck(cudaMemcpyAsync(b, s.rhs.p, (size_t)n3 * nrhs * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "x copy");
    r.sync("bhm_solve");
    if (s.precision == BGPU_MIXED && s.mixed)
      for (auto& line : s.mixed->profile_report()) note("%s", line.c_str());
    if (s.precision == BGPU_HMATRIX)
      note("solve: %d right-hand sides by GMRES on the H-matrix, %d steps, relative residual %.1e, %.2f ms", nrhs,
           (int)g_solve_info[0], g_solve_info[1], r.ms[3]);
    else if (s.precision == BGPU_MIXED && s.mixed)
      note("solve: %d right-hand sides, %d refinement steps, relative residual %.1e, %.2f ms", nrhs,
          (int)g_solve_info[0], g_solve_info[1], r.ms[3]);
    else
      note("solve: %d right-hand sides with the FP64 LU factors, %.2f ms", nrhs, r.ms[3]);
    return 0;
  });
}

int bhm_log_line(char* buf, int len) { return g_messages.take(buf, len); }

void bhm_destroy(void) {
  g.reset();
  g_rt.reset();
}

// ---------------------------------------------------------------------------------------------
// best_gpu.h
// ---------------------------------------------------------------------------------------------

int bgpu_set_precision(int mode) {
  if (mode != -1 && mode != BGPU_FP64 && mode != BGPU_MIXED && mode != BGPU_HMATRIX) {
    note("error: unknown precision %d", mode);
    return 1;
  }
  g_prec_override = mode;
  return 0;
}

int bgpu_precision(void) { return g ? g->precision : -1; }

int bgpu_set_refinement(int max_restarts, int krylov) {
  if (max_restarts < 0 || krylov < 1 || krylov > 16) {
    note("error: bgpu_set_refinement: restarts >= 0 and 1 <= krylov <= 16");
    return 1;
  }
  g_refine[0] = max_restarts;
  g_refine[1] = krylov;
  if (g && g->mixed) g->mixed->set_refinement(max_restarts, krylov);
  return 0;
}

int bgpu_series_create(int count, const int* n, const double* v1, const double* v2, const double* v3,
                       const double* area, const double* afac, double cg) {
  return status_of([&] {
    if (count < 1 || count > kMaxSeries) {
      note("error: bgpu_series_create: %d meshes (1 to %d)", count, kMaxSeries);
      return 1;
    }
    for (int i = 0; i < count; ++i)
      if (n[i] < 1) {
        note("error: bgpu_series_create: mesh %d has no triangles", i);
        return 1;
      }
    Runtime& r = rt();
    g_series.reset();
    auto S = std::make_unique<Series>();
    S->count = count;
    S->cg = cg;
    long tot = 0;
    for (int i = 0; i < count; ++i) {
      S->n.push_back(n[i]);
      S->t0.push_back(tot);
      S->afac.push_back(afac[i]);
      tot += n[i];
    }
    std::vector<double> h;
    h.reserve((size_t)tot * kGeoStride);
    for (int i = 0; i < count; ++i) {
      const long o = S->t0[i];
      std::vector<double> g = geo_host(n[i], v1 + 3 * o, v2 + 3 * o, v3 + 3 * o, area + o);
      h.insert(h.end(), g.begin(), g.end());
      S->fast_ok.push_back(mesh_fast_ok(v1 + 3 * o, n[i], 1, n[i]) && mesh_fast_ok(v2 + 3 * o, n[i], 1, n[i]) &&
                           mesh_fast_ok(v3 + 3 * o, n[i], 1, n[i]));
    }
    S->geo.ensure(h.size() * sizeof(double), "series meshes");
    S->xc.ensure((size_t)tot * kXcStride * sizeof(double), "series incenters");
    S->self9.ensure((size_t)tot * 9 * sizeof(double), "series self blocks");
    S->diag.ensure(sizeof(double) * count, "series diagonal means");
    ck(cudaMemcpyAsync(S->geo.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, r.stream), "mesh copy");
    for (int i = 0; i < count; ++i) {
      ck(launch_self_blocks(S->mesh(i), r.stream), "self blocks");
      ck(launch_diag_mean(S->mesh(i), S->diag.as<double>() + i, r.stream), "diagonal mean");
    }
    std::vector<double> xc((size_t)tot * kXcStride);
    ck(cudaMemcpyAsync(xc.data(), S->xc.p, xc.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream),
       "incenter copy");
    r.sync("bgpu_series_create");
    S->x_host.resize((size_t)3 * tot);
    for (int i = 0; i < count; ++i)
      for (int t = 0; t < n[i]; ++t)
        for (int c = 0; c < 3; ++c)
          S->x_host[3 * S->t0[i] + (size_t)c * n[i] + t] = xc[(size_t)(S->t0[i] + t) * kXcStride + c];
    g_series = std::move(S);
    return 0;
  });
}

int bgpu_series_incenters(double* x) {
  return status_of([&] {
    Series& S = series();
    std::memcpy(x, S.x_host.data(), S.x_host.size() * sizeof(double));
    return 0;
  });
}

int bgpu_series_diag_mean(double* dm) {
  return status_of([&] {
    Series& S = series();
    Runtime& r = rt();
    ck(cudaMemcpyAsync(dm, S.diag.p, sizeof(double) * S.count, cudaMemcpyDeviceToHost, r.stream), "diag copy");
    r.sync("bgpu_series_diag_mean");
    return 0;
  });
}

int bgpu_series_build(const int* ndef, const double* gdef, const int* comp, const double* xmu, int tune) {
  return status_of([&] {
    Series& S = series();
    Runtime& r = rt();
    S.factored = false;
    const long tot = S.t0[S.count - 1] + S.n[S.count - 1];
    // deflation data
    S.ndef.assign(ndef, ndef + S.count);
    S.gdef0.clear();
    long ng = 0;
    bool any_comp = false;
    for (int i = 0; i < S.count; ++i) {
      S.gdef0.push_back(ng);
      ng += std::max(0, S.ndef[i]);
      any_comp = any_comp || S.ndef[i] > 1;
    }
    if (ng > 0) {
      S.gdef.ensure(sizeof(double) * ng, "deflation weights");
      S.xmu.ensure(sizeof(double) * 3 * tot, "deflation vectors");
      ck(cudaMemcpyAsync(S.gdef.p, gdef, sizeof(double) * ng, cudaMemcpyHostToDevice, r.stream), "gdef copy");
      ck(cudaMemcpyAsync(S.xmu.p, xmu, sizeof(double) * 3 * tot, cudaMemcpyHostToDevice, r.stream), "xmu copy");
    }
    if (any_comp) {
      S.comp.ensure(sizeof(int) * tot, "surface labels");
      ck(cudaMemcpyAsync(S.comp.p, comp, sizeof(int) * tot, cudaMemcpyHostToDevice, r.stream), "comp copy");
    }
    // matrices and factors
    if (S.gr0.empty()) {
      size_t g0 = 0, i0 = 0;
      for (int i = 0; i < S.count; ++i) {
        const int n3 = 3 * S.n[i];
        S.ld.push_back(padded_ld(n3));
        S.gr0.push_back(g0);
        S.inv0.push_back(i0);
        g0 += (size_t)S.ld[i] * n3;
        i0 += diag_inverse_elems(n3);
      }
      S.gr.ensure(g0 * sizeof(double), "series GR (FP64)");
      S.dl.ensure(i0 * sizeof(double), "diagonal-block inverses (L)");
      S.du.ensure(i0 * sizeof(double), "diagonal-block inverses (U)");
      S.ipiv.ensure(sizeof(int) * 3 * tot, "pivots");
      S.perm.ensure(sizeof(int) * 3 * tot, "permutations");
      S.info.ensure(sizeof(int) * kMaxSeries, "info", true);
    }
    if (S.precision == BGPU_MIXED) {
      try {
        series_build_mixed(S, r);
        r.sync("bgpu_series_build");
        S.ms[0] = r.elapsed(2, 4);
        S.ms[1] = 0;
        S.built_precision = BGPU_MIXED;
        S.factored = true;
        note("GPU series build: %d meshes (N = %d .. %d), mixed precision (BF16 tensor-core LU per mesh, one stream "
             "each), %.1f ms", S.count, *std::min_element(S.n.begin(), S.n.end()),
             *std::max_element(S.n.begin(), S.n.end()), S.ms[0]);
        return 0;
      } catch (const MixedFailure& e) {
        note("series, mixed precision: %s; building the FP64 series instead", e.what());
      }
    }
    S.built_precision = BGPU_FP64;
    ck(lu_prepare(), "LU kernel attributes");
    if (tune) {
      // a first build with the DGEMM autotuner on (direct launches; the result is overwritten below)
      ck(cudaEventRecord(r.ev[0], r.stream), "event");
      lu_autotune(true);
      try {
        series_record(S, r, r.stream, r.ev[3]);
      } catch (...) {
        lu_autotune(false);
        throw;
      }
      lu_autotune(false);
      ck(cudaEventRecord(r.ev[1], r.stream), "event");
      r.check_status("series tuning");
      S.ms[3] = r.elapsed(0, 1);
      S.ms[1] = r.elapsed(0, 3);
      std::string table = lu_autotune_table();
      size_t a = 0;
      while (a < table.size()) {
        size_t b = table.find('\n', a);
        if (b == std::string::npos) b = table.size();
        note("autotune: %s", table.substr(a, b - a).c_str());
        a = b + 1;
      }
      if (S.graph) {  // shapes may have changed: capture again
        cudaGraphExecDestroy(S.graph);
        S.graph = nullptr;
        S.graph_tried = false;
      }
    }
    if (!S.graph && !S.graph_tried) {
      S.graph_tried = true;
      cudaStream_t cs;
      ck(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
      cudaGraph_t gph = nullptr;
      const unsigned long long launches0 = g_launches;
      bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      std::string why;
      if (ok) {
        try {
          series_record(S, r, cs);
        } catch (const std::exception& e) {
          why = e.what();
          ok = false;
        }
        if (cudaStreamEndCapture(cs, &gph) != cudaSuccess) ok = false;
      }
      const unsigned long long captured = g_launches - launches0;
      g_launches = launches0;
      if (ok && gph && cudaGraphInstantiate(&S.graph, gph, 0) == cudaSuccess) {
        S.graph_kernels = captured;
      } else {
        S.graph = nullptr;
        note("series: graph capture unavailable (%s); launching directly", why.empty() ? "capture failed" : why.c_str());
      }
      if (gph) cudaGraphDestroy(gph);
      cudaGetLastError();
      cudaStreamDestroy(cs);
    }
    ck(cudaEventRecord(r.ev[2], r.stream), "event");
    if (S.graph) {
      ck(cudaGraphLaunch(S.graph, r.stream), "series graph");
      g_launches += S.graph_kernels;
    } else {
      series_record(S, r, r.stream, r.ev[3]);
    }
    ck(cudaEventRecord(r.ev[4], r.stream), "event");
    r.check_status("bgpu_series_build");
    S.ms[0] = r.elapsed(2, 4);
    if (!S.graph) S.ms[1] = r.elapsed(2, 3);
    std::vector<int> info(S.count);
    ck(cudaMemcpy(info.data(), S.info.p, sizeof(int) * S.count, cudaMemcpyDeviceToHost), "info read");
    for (int i = 0; i < S.count; ++i)
      if (info[i] > 0) {
        note("error: series mesh %d: the LU factorisation found U(%d,%d) = 0: GR is singular", i, info[i], info[i]);
        return 1;
      }
    S.factored = true;
    note("GPU series build: %d meshes (N = %d .. %d), %s, %.1f ms", S.count, *std::min_element(S.n.begin(), S.n.end()),
        *std::max_element(S.n.begin(), S.n.end()), S.graph ? "one CUDA graph" : "direct launches", S.ms[0]);
    return 0;
  });
}

int bgpu_series_solve(int nrhs, double* b) {
  return status_of([&] {
    Series& S = series();
    Runtime& r = rt();
    if (!S.factored) throw std::runtime_error("bgpu_series_build has not factored the series");
    if (nrhs <= 0) return 0;
    const long rows = S.rows();
    S.rhs.ensure((size_t)rows * nrhs * sizeof(double), "series right-hand sides");
    ck(cudaMemcpyAsync(S.rhs.p, b, (size_t)rows * nrhs * sizeof(double), cudaMemcpyHostToDevice, r.stream), "b copy");
    ck(cudaEventRecord(r.ev[5], r.stream), "event");
    if (S.built_precision == BGPU_MIXED) {
      MixedReport rep;
      for (int i = 0; i < S.count; ++i) {
        double* bi = S.rhs.as<double>() + (size_t)3 * S.t0[i] * nrhs;
        ck(cudaEventRecord(r.ev[7], r.stream), "event");
        ck(cudaStreamWaitEvent(S.streams[i], r.ev[7], 0), "series fork");
        S.mixed[i]->solve(nrhs, bi, 3L * S.n[i], S.streams[i], &rep);
        ck(cudaEventRecord(S.ev_done[i], S.streams[i]), "event");
        ck(cudaStreamWaitEvent(r.stream, S.ev_done[i], 0), "series join");
      }
      ck(cudaEventRecord(r.ev[6], r.stream), "event");
      ck(cudaMemcpyAsync(b, S.rhs.p, (size_t)rows * nrhs * sizeof(double), cudaMemcpyDeviceToHost, r.stream),
         "x copy");
      r.check_status("bgpu_series_solve");
      S.ms[2] = r.elapsed(5, 6);
      return 0;
    }
    long maxn = 0;
    for (int i = 0; i < S.count; ++i) maxn = std::max<long>(maxn, 3L * S.n[i]);
    r.ensure_trsv((int)maxn);
    for (int i = 0; i < S.count; ++i) {
      const int n3 = 3 * S.n[i];
      double* bi = S.rhs.as<double>() + (size_t)3 * S.t0[i] * nrhs;
      for (int c = 0; c < nrhs; c += 16) {
        const int q = std::min(16, nrhs - c);
        ck(getrs64_inv(S.gr.as<double>() + S.gr0[i], S.ld[i], S.dl.as<double>() + S.inv0[i],
                       S.du.as<double>() + S.inv0[i], n3, S.perm.as<int>() + 3 * S.t0[i], bi + (size_t)c * n3, n3, q,
                       r.trsv_scratch.p, r.status.as<int>(), r.stream),
           "series solve");
      }
      ck(check_finite(bi, n3, n3, nrhs, r.status.as<int>(), r.stream), "finite check");
    }
    ck(cudaEventRecord(r.ev[6], r.stream), "event");
    ck(cudaMemcpyAsync(b, S.rhs.p, (size_t)rows * nrhs * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "x copy");
    r.check_status("bgpu_series_solve");
    S.ms[2] = r.elapsed(5, 6);
    return 0;
  });
}

int bgpu_series_timings(double* ms, int len) {
  if (!g_series) return 0;
  const int k = std::min(len, 4);
  for (int i = 0; i < k; ++i) ms[i] = g_series->ms[i];
  return k;
}

int bgpu_series_set_precision(int mode) {
  return status_of([&] {
    Series& S = series();
    if (mode != BGPU_FP64 && mode != BGPU_MIXED) {
      note("error: bgpu_series_set_precision: mode %d is neither BGPU_FP64 nor BGPU_MIXED", mode);
      return 1;
    }
    S.precision = mode;
    return 0;
  });
}

void bgpu_series_destroy(void) { g_series.reset(); }

int bgpu_autotune_table(char* buf, int len) {
  const std::string t = lu_autotune_table();
  if (len <= 0) return (int)t.size();
  const int k = std::min<int>(len - 1, (int)t.size());
  std::memcpy(buf, t.data(), k);
  buf[k] = 0;
  return (int)t.size();
}

int bgpu_best_gradient(int iarea, double truearea, double wm, double* values, double* grad) {
  return status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    if (!s.factored || s.precision != BGPU_FP64) {
      note("error: bgpu_best_gradient needs the FP64 LU of the last bhm_build (direct = 1, or "
          "bgpu_set_precision(BGPU_FP64))");
      return 1;
    }
    const int n = s.n;
    const size_t n3 = 3 * (size_t)n;
    const double* x = s.x_host.data();
    const double* area = s.area_host.data();
    const double cg = s.cg, afac = s.afac;
    constexpr int K = 3, C = 17;  // results D_t, D_r, [eta]; adjoint columns 6 + 6 + 5
    using Clock = std::chrono::steady_clock;
    const auto h0 = Clock::now();
    auto since = [&](Clock::time_point a) { return std::chrono::duration<double, std::milli>(Clock::now() - a).count(); };
    double hms[6] = {};
    ck(cudaEventRecord(r.ev[0], r.stream), "event");
    // 1. the solutions of the six flows and the five strain flows (best/difco.f:28-44, visco.f:216-243)
    std::vector<double> F(n3 * 11);
    bgpu_best_rhs6(n, x, F.data());
    bgpu_best_strain5(n, x, F.data() + 6 * n3);
    DevBuf dF;
    dF.ensure(F.size() * sizeof(double), "gradient right-hand sides");
    ck(cudaMemcpyAsync(dF.p, F.data(), F.size() * sizeof(double), cudaMemcpyHostToDevice, r.stream), "b copy");
    solve_device(s, r, 11, dF.as<double>(), (long)n3);
    ck(cudaMemcpyAsync(F.data(), dF.p, F.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "x copy");
    r.sync("gradient solve");
    hms[0] = since(h0);
    auto fv = [&](int col, int t, int c) { return F[(size_t)col * n3 + 3 * (size_t)t + c]; };
    auto xv = [&](int t, int c) { return x[(size_t)c * n + t]; };
    // 2. the results and their seeds: d/dF, d/dX and d/d(area) of the post-processing
    double tens[60], tr[4], vis[4];
    bgpu_best_difco(n, x, area, cg, F.data(), tens);
    bgpu_best_traces(tens, tr);
    bgpu_best_visco(n, x, area, cg, 0, F.data() + 6 * n3, F.data(), vis);
    const double eta_f = wm > 0 ? 0.602214 / wm : 1.0;
    values[0] = tr[2];
    values[1] = tr[3];
    values[2] = vis[0] * eta_f;
    double Kraw[4][9] = {};
    for (int mx = 0; mx < 6; ++mx) {
      const int i = mx % 3, bf = mx < 3 ? 0 : 2;
      for (int t = 0; t < n; ++t) {
        const double F1 = fv(mx, t, 0), F2 = fv(mx, t, 1), F3 = fv(mx, t, 2), X = xv(t, 0), Y = xv(t, 1), Z = xv(t, 2);
        const double T[3] = {Y * F3 - Z * F2, Z * F1 - X * F3, X * F2 - Y * F1}, Fv[3] = {F1, F2, F3};
        for (int j = 0; j < 3; ++j) {
          Kraw[bf][3 * j + i] += area[t] * Fv[j];
          Kraw[bf + 1][3 * j + i] += area[t] * T[j];
        }
      }
    }
    double gK[2][4][9];
    difco_post_gradient(Kraw, cg, gK[0], gK[1]);
    std::vector<double> Fbar(n3 * C, 0.0), Xbar((size_t)K * n * 3, 0.0), Abar((size_t)K * n, 0.0);
    auto XB = [&](int k, int t, int c) -> double& { return Xbar[((size_t)k * n + t) * 3 + c]; };
    for (int k = 0; k < 2; ++k)
      for (int mx = 0; mx < 6; ++mx) {
        const int i = mx % 3, bf = mx < 3 ? 0 : 2;
        const double gF[3] = {gK[k][bf][i], gK[k][bf][3 + i], gK[k][bf][6 + i]};
        const double gT[3] = {gK[k][bf + 1][i], gK[k][bf + 1][3 + i], gK[k][bf + 1][6 + i]};
        for (int t = 0; t < n; ++t) {
          const double f[3] = {fv(mx, t, 0), fv(mx, t, 1), fv(mx, t, 2)}, X[3] = {xv(t, 0), xv(t, 1), xv(t, 2)};
          const double A = area[t];
          // K += A F (forces), A X x F (torques)
          const double TxX[3] = {gT[1] * X[2] - gT[2] * X[1], gT[2] * X[0] - gT[0] * X[2], gT[0] * X[1] - gT[1] * X[0]};
          const double FxT[3] = {f[1] * gT[2] - f[2] * gT[1], f[2] * gT[0] - f[0] * gT[2], f[0] * gT[1] - f[1] * gT[0]};
          const double XxF[3] = {X[1] * f[2] - X[2] * f[1], X[2] * f[0] - X[0] * f[2], X[0] * f[1] - X[1] * f[0]};
          for (int c = 0; c < 3; ++c) {
            Fbar[(size_t)(6 * k + mx) * n3 + 3 * (size_t)t + c] = A * (gF[c] + TxX[c]);
            XB(k, t, c) += A * FxT[c];
          }
          Abar[(size_t)k * n + t] += f[0] * gF[0] + f[1] * gF[1] + f[2] * gF[2] + XxF[0] * gT[0] + XxF[1] * gT[1] +
                                     XxF[2] * gT[2];
        }
      }
    {
      // CHI' (best/visco.f:192-213 with icov = 0) is linear in the strain solutions: per column l and
      // component c, the coordinate it is multiplied by and its coefficient
      const double pi = 3.1415926535897932385;
      const double f8 = eta_f * 8 * pi * (cg == 0 ? 0.75 : 1.0);
      const int xi[5][3] = {{1, 0, -1}, {2, -1, 0}, {-1, 2, 1}, {0, 1, 2}, {0, 1, 2}};
      const double cf[5][3] = {{0.1, 0.1, 0}, {0.1, 0, 0.1}, {0, 0.1, 0.1}, {1 / 15., -2 / 15., 1 / 15.},
                               {1 / 15., 1 / 15., -2 / 15.}};
      for (int l = 0; l < 5; ++l)
        for (int c = 0; c < 3; ++c) {
          if (xi[l][c] < 0) continue;
          const double co = f8 * cf[l][c];
          for (int t = 0; t < n; ++t) {
            const double A = area[t], X = xv(t, xi[l][c]), V = fv(6 + l, t, c);
            Fbar[(size_t)(12 + l) * n3 + 3 * (size_t)t + c] = co * A * X;
            XB(2, t, xi[l][c]) += co * A * V;
            Abar[2 * (size_t)n + t] += co * V * X;
          }
        }
    }
    hms[1] = since(h0);
    // 3. the adjoint solve, lambda = GR^-T dJ/dF, with the same LU
    DevBuf dL;
    dL.ensure(Fbar.size() * sizeof(double), "adjoint vectors");
    ck(cudaMemcpyAsync(dL.p, Fbar.data(), Fbar.size() * sizeof(double), cudaMemcpyHostToDevice, r.stream), "copy");
    r.ensure_trsv(3 * n);
    for (int c = 0; c < C; c += 16) {
      const int q = std::min(16, C - c);
      ck(getrs64_trans_inv(s.gr.as<double>(), s.ld, s.dl64.as<double>(), s.du64.as<double>(), (int)n3, s.perm.as<int>(),
                           dL.as<double>() + (size_t)c * n3, (long)n3, q, r.trsv_scratch.p, r.status.as<int>(),
                           r.stream),
         "adjoint solve");
    }
    std::vector<double> lam(n3 * C);
    ck(cudaMemcpyAsync(lam.data(), dL.p, lam.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "copy");
    r.check_status("adjoint solve");
    hms[2] = since(h0);
    auto lv = [&](int col, int t, int c) { return lam[(size_t)col * n3 + 3 * (size_t)t + c]; };
    // the F column each adjoint column pairs with, and its result
    int fcol[C], cout_[C];
    for (int c = 0; c < C; ++c) {
      fcol[c] = c < 6 ? c : (c < 12 ? c - 6 : 6 + (c - 12));
      cout_[c] = c < 6 ? 0 : (c < 12 ? 1 : 2);
    }
    // 4. the right-hand sides' dependence on the incenters: rotations e_i x X, strains
    for (int k = 0; k < 2; ++k)
      for (int t = 0; t < n; ++t)
        for (int i = 0; i < 3; ++i) {
          const double a0 = lv(6 * k + 3 + i, t, 0), a1 = lv(6 * k + 3 + i, t, 1), a2 = lv(6 * k + 3 + i, t, 2);
          // lambda . (e_i x dX) = dX . (lambda x e_i)
          const double ax[3][3] = {{0.0, a2, -a1}, {-a2, 0.0, a0}, {a1, -a0, 0.0}};
          for (int c = 0; c < 3; ++c) XB(k, t, c) += ax[i][c];
        }
    for (int t = 0; t < n; ++t) {
      const int b = 12;
      XB(2, t, 1) += 0.5 * lv(b + 0, t, 0);
      XB(2, t, 0) += 0.5 * lv(b + 0, t, 1);
      XB(2, t, 2) += 0.5 * lv(b + 1, t, 0);
      XB(2, t, 0) += 0.5 * lv(b + 1, t, 2);
      XB(2, t, 2) += 0.5 * lv(b + 2, t, 1);
      XB(2, t, 1) += 0.5 * lv(b + 2, t, 2);
      XB(2, t, 0) += 0.5 * lv(b + 3, t, 0);
      XB(2, t, 1) -= 0.5 * lv(b + 3, t, 1);
      XB(2, t, 0) += 0.5 * lv(b + 4, t, 0);
      XB(2, t, 2) -= 0.5 * lv(b + 4, t, 2);
    }
    // 5. the pair integrals' adjoint on the GPU (GR recomputed, contracted on the fly)
    std::vector<double> lamT(n3 * C), fsT(n3 * C);
    for (int t = 0; t < n; ++t)
      for (int c = 0; c < C; ++c)
        for (int a = 0; a < 3; ++a) {
          lamT[((size_t)t * C + c) * 3 + a] = lv(c, t, a);
          fsT[((size_t)t * C + c) * 3 + a] = fv(fcol[c], t, a);
        }
    DevBuf dlamT, dfsT, dxb, dqb, dscr;
    dlamT.ensure(lamT.size() * sizeof(double), "adjoint vectors (by triangle)");
    dfsT.ensure(fsT.size() * sizeof(double), "solutions (by triangle)");
    dxb.ensure((size_t)n * 3 * K * sizeof(double), "incenter gradients");
    dqb.ensure((size_t)n * 10 * K * sizeof(double), "corner gradients");
    dscr.ensure(pair_adjoint_scratch_bytes(n, K), "adjoint partial sums");
    ck(cudaMemcpyAsync(dlamT.p, lamT.data(), lamT.size() * sizeof(double), cudaMemcpyHostToDevice, r.stream), "copy");
    ck(cudaMemcpyAsync(dfsT.p, fsT.data(), fsT.size() * sizeof(double), cudaMemcpyHostToDevice, r.stream), "copy");
    ck(cudaEventRecord(r.ev[1], r.stream), "event");
    ck(launch_pair_adjoint(s.mesh(), K, dlamT.as<double>(), dfsT.as<double>(), C, cout_, dxb.as<double>(),
                           dqb.as<double>(), dscr.p, r.stream),
       "pair adjoint");
    ck(cudaEventRecord(r.ev[2], r.stream), "event");
    std::vector<double> xb((size_t)n * 3 * K), qb((size_t)n * 10 * K), self9((size_t)n * 9);
    ck(cudaMemcpyAsync(xb.data(), dxb.p, xb.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "copy");
    ck(cudaMemcpyAsync(qb.data(), dqb.p, qb.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "copy");
    ck(cudaMemcpyAsync(self9.data(), s.self9.p, self9.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream),
       "copy");
    r.check_status("pair adjoint");
    r.ms[5] = r.elapsed(1, 2);
    hms[3] = since(h0);
    for (int k = 0; k < K; ++k)
      for (int t = 0; t < n; ++t) {
        for (int c = 0; c < 3; ++c) XB(k, t, c) += xb[(size_t)t * 3 * K + 3 * k + c];
        Abar[(size_t)k * n + t] += qb[(size_t)t * 10 * K + 10 * k + 9];
      }
    // 6. the self blocks' weights
    std::vector<double> Ws((size_t)K * n * 9, 0.0);
    for (int c = 0; c < C; ++c)
      for (int t = 0; t < n; ++t)
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b)
            Ws[((size_t)cout_[c] * n + t) * 9 + 3 * a + b] -= lv(c, t, a) * fv(fcol[c], t, b);
    // 7. the deflation (best/best.f:406-425): GR += GDEF_d XMU XMU^T on each surface d, GDEF_d =
    // DIAGM / |XMU_d|^2, XMU = area * unit normal, DIAGM the mean of the self blocks' diagonals
    std::vector<double> nbar((size_t)K * n * 3, 0.0);
    if (s.ndef >= 1) {
      const int nd = s.ndef;
      auto surf = [&](int t) { return nd > 1 ? s.comp_host[t] - 1 : 0; };
      const double* xmu = s.xmu_host.data();
      std::vector<double> Q(nd, 0.0);
      for (int t = 0; t < n; ++t)
        Q[surf(t)] += xmu[3 * t] * xmu[3 * t] + xmu[3 * t + 1] * xmu[3 * t + 1] + xmu[3 * t + 2] * xmu[3 * t + 2];
      const double diagm = s.gdef_host[0] * Q[0];
      std::vector<double> xmub((size_t)K * n3, 0.0);
      for (int k = 0; k < K; ++k) {
        std::vector<double> gG(nd, 0.0);
        for (int c = 0; c < C; ++c) {
          if (cout_[c] != k) continue;
          std::vector<double> u(nd, 0.0), w(nd, 0.0);
          for (int t = 0; t < n; ++t)
            for (int a = 0; a < 3; ++a) {
              u[surf(t)] += lv(c, t, a) * xmu[3 * t + a];
              w[surf(t)] += xmu[3 * t + a] * fv(fcol[c], t, a);
            }
          for (int d = 0; d < nd; ++d) gG[d] -= u[d] * w[d];
          for (int t = 0; t < n; ++t) {
            const int d = surf(t);
            for (int a = 0; a < 3; ++a)
              xmub[(size_t)k * n3 + 3 * t + a] -= s.gdef_host[d] * (lv(c, t, a) * w[d] + fv(fcol[c], t, a) * u[d]);
          }
        }
        double gdiag = 0.0;
        for (int d = 0; d < nd; ++d) {
          gdiag += gG[d] / Q[d];
          const double gQ = -gG[d] * diagm / (Q[d] * Q[d]);
          for (int t = 0; t < n; ++t)
            if (surf(t) == d)
              for (int a = 0; a < 3; ++a) xmub[(size_t)k * n3 + 3 * t + a] += 2.0 * gQ * xmu[3 * t + a];
        }
        for (int t = 0; t < n; ++t)
          for (int a = 0; a < 3; ++a) Ws[((size_t)k * n + t) * 9 + 4 * a] += gdiag / (double)n3;
        // XMU_t = area_t * unit normal_t
        for (int t = 0; t < n; ++t) {
          double dotp = 0.0;
          for (int a = 0; a < 3; ++a) {
            const double nh = xmu[3 * t + a] / area[t];
            dotp += xmub[(size_t)k * n3 + 3 * t + a] * nh;
            nbar[((size_t)k * n + t) * 3 + a] = area[t] * xmub[(size_t)k * n3 + 3 * t + a];
          }
          Abar[(size_t)k * n + t] += dotp;
        }
      }
    }
    // 8. corrected area = AFAC * raw area; AFAC = TRUEAREA / total raw area when iarea (best.f:286-298);
    // the self blocks scale with sqrt(AFAC) (tgetgr.f:106)
    double totraw = 0.0;
    for (int t = 0; t < n; ++t) totraw += area[t] / afac;
    std::vector<double> cot((size_t)n * K * 16, 0.0);
    for (int k = 0; k < K; ++k) {
      double gafac = 0.0;
      if (iarea) {
        for (int t = 0; t < n; ++t) {
          gafac += (area[t] / afac) * Abar[(size_t)k * n + t];
          for (int e = 0; e < 9; ++e) gafac += Ws[((size_t)k * n + t) * 9 + e] * self9[9 * (size_t)t + e] / (2.0 * afac);
        }
      }
      const double gtot = iarea ? -gafac * afac / totraw : 0.0;
      for (int t = 0; t < n; ++t) {
        double* ct = cot.data() + ((size_t)t * K + k) * 16;
        for (int e = 0; e < 9; ++e) ct[e] = Ws[((size_t)k * n + t) * 9 + e];
        for (int c = 0; c < 3; ++c) ct[9 + c] = XB(k, t, c);
        ct[12] = afac * Abar[(size_t)k * n + t] + gtot;
        for (int c = 0; c < 3; ++c) ct[13 + c] = nbar[((size_t)k * n + t) * 3 + c];
      }
    }
    // 9. the per-triangle geometry's adjoint on the GPU
    DevBuf dcot, dvb;
    dcot.ensure(cot.size() * sizeof(double), "triangle cotangents");
    dvb.ensure((size_t)n * K * 9 * sizeof(double), "triangle gradients");
    ck(cudaMemcpyAsync(dcot.p, cot.data(), cot.size() * sizeof(double), cudaMemcpyHostToDevice, r.stream), "copy");
    ck(launch_tri_adjoint(s.mesh(), K, dcot.as<double>(), dvb.as<double>(), r.stream), "triangle adjoint");
    std::vector<double> vb((size_t)n * K * 9);
    ck(cudaMemcpyAsync(vb.data(), dvb.p, vb.size() * sizeof(double), cudaMemcpyDeviceToHost, r.stream), "copy");
    ck(cudaEventRecord(r.ev[3], r.stream), "event");
    hms[4] = since(h0);
    r.check_status("triangle adjoint");
    r.ms[6] = r.elapsed(0, 3);
    // 10. the corners as given: the centroid of the triangle centroids is subtracted first
    // (best.f:261-272), so every corner's gradient loses the mean over all corners
    for (int k = 0; k < K; ++k) {
      double mean[3] = {0, 0, 0};
      for (int t = 0; t < n; ++t)
        for (int corner = 0; corner < 3; ++corner)
          for (int c = 0; c < 3; ++c) {
            const double g = vb[((size_t)t * K + k) * 9 + 3 * corner + c] + qb[(size_t)t * 10 * K + 10 * k + 3 * corner + c];
            grad[(size_t)k * 9 * n + (size_t)corner * 3 * n + (size_t)c * n + t] = g;
            mean[c] += g;
          }
      for (int c = 0; c < 3; ++c) mean[c] /= 3.0 * n;
      for (int corner = 0; corner < 3; ++corner)
        for (int c = 0; c < 3; ++c)
          for (int t = 0; t < n; ++t) grad[(size_t)k * 9 * n + (size_t)corner * 3 * n + (size_t)c * n + t] -= mean[c];
    }
    hms[5] = since(h0);
    note("gradient: D_t %.6e, D_r %.6e, %s %.6e; pair adjoint %.1f ms (GPU); host clock: solves %.1f, seeds %.1f, "
        "adjoint solve %.1f, pair adjoint %.1f, deflation/area/triangles %.1f, total %.1f ms",
        values[0], values[1], wm > 0 ? "[eta]" : "CHI'", values[2], r.ms[5], hms[0], hms[1] - hms[0], hms[2] - hms[1],
        hms[3] - hms[2], hms[4] - hms[3], hms[5]);
    return 0;
  });
}

int bgpu_hmatrix_set_options(int leaf, double eta, int kmax) {
  return status_of([&] {
    HMatrixSolver probe;
    probe.set_options(leaf, eta, kmax);  // validates
    g_hm_opts.leaf = leaf;
    g_hm_opts.eta = eta;
    g_hm_opts.kmax = kmax;
    return 0;
  });
}

int bgpu_hmatrix_stats(double* out, int len) {
  return status_of([&] {
    Solver& s = solver();
    if (!s.hmat) throw std::runtime_error("bgpu_hmatrix_stats: the last bhm_build did not take the H-matrix path");
    const std::vector<double> st = s.hmat->stats();
    for (int i = 0; i < len && i < (int)st.size(); ++i) out[i] = st[i];
    return 0;
  });
}

int bgpu_hmatrix_matvec_device(int nrhs, const double* d_x, int ldx, double* d_y, int ldy) {
  return status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    if (!s.hmat || s.precision != BGPU_HMATRIX)
      throw std::runtime_error("bgpu_hmatrix_matvec_device: the last bhm_build did not take the H-matrix path");
    if (nrhs < 0 || ldx < 3 * s.n || ldy < 3 * s.n) throw std::runtime_error("bgpu_hmatrix_matvec_device: bad sizes");
    try {
      s.hmat->matvec(nrhs, d_x, ldx, d_y, ldy, r.stream);
    } catch (const std::runtime_error& e) {
      throw CudaError(e.what());
    }
    r.sync("bgpu_hmatrix_matvec_device");
    return 0;
  });
}

int bgpu_hmatrix_plan(int n, const double* x, const double* v1, const double* v2, const double* v3, int leaf,
                      double eta, int kmax, int* perm, int* counts) {
  return status_of([&] {
    if (n < 1) throw std::runtime_error("bgpu_hmatrix_plan: n < 1");
    std::vector<double> geo((size_t)n * kGeoStride, 0.0), xc((size_t)n * kXcStride, 0.0);
    for (int t = 0; t < n; ++t)
      for (int c = 0; c < 3; ++c) {
        geo[(size_t)t * kGeoStride + c] = v1[(size_t)c * n + t];
        geo[(size_t)t * kGeoStride + 3 + c] = v2[(size_t)c * n + t];
        geo[(size_t)t * kGeoStride + 6 + c] = v3[(size_t)c * n + t];
        xc[(size_t)t * kXcStride + c] = x[(size_t)c * n + t];
      }
    const HPlan p = hplan_build(n, geo.data(), xc.data(), leaf, eta, kmax);
    for (int k = 0; k < n; ++k) perm[k] = p.perm[k];
    int nd = 0, nl = 0, na = 0;
    for (const auto& b : p.blocks) {
      nd += !b.lowrank;
      nl += b.lowrank;
      na += b.admissible;
    }
    counts[0] = p.depth;
    counts[1] = (int)p.leaves.size();
    counts[2] = nd;
    counts[3] = nl;
    counts[4] = na;
    return 0;
  });
}

int bgpu_timings(double* ms, int len) {
  if (!g_rt) return 0;
  double v[7] = {g_rt->ms[0], g_rt->ms[1], g_rt->ms[2], g_rt->ms[3], g_rt->ms[4], g_solve_info[0], g_solve_info[1]};
  const int k = std::min(len, 7);
  for (int i = 0; i < k; ++i) ms[i] = v[i];
  return k;
}

void* bgpu_stream(void) {
  void* p = nullptr;
  status_of([&] {
    p = (void*)rt().stream;
    return 0;
  });
  return p;
}

int bgpu_solve_device(int nrhs, double* d_b, int ldb) {
  return status_of([&] {
    solve_device(solver(), rt(), nrhs, d_b, ldb);
    return 0;
  });
}

int bgpu_dgetrf_device(int n, double* d_a, int lda, int* d_ipiv, int* info) {
  return status_of([&] {
    Runtime& r = rt();
    if (n < 0 || lda < std::max(1, n) || (lda & 1) || ((uintptr_t)d_a & 15)) {
      note("error: bgpu_dgetrf_device needs lda >= n, lda even and a 16-byte aligned matrix");
      return 1;
    }
    LuScratch ws{r.lu_scratch.p, r.lu_scratch.bytes};
    ck(cudaEventRecord(r.ev[3], r.stream), "event");
    ck(lu64_getrf(d_a, lda, n, d_ipiv, r.info.as<int>(), r.status.as<int>(), ws, r.stream), "LU");
    ck(cudaEventRecord(r.ev[5], r.stream), "event");
    r.check_status("dgetrf");
    ck(cudaMemcpy(info, r.info.p, sizeof(int), cudaMemcpyDeviceToHost), "info read");
    r.ms[2] = r.elapsed(3, 5);
    return 0;
  });
}

int bgpu_dgetrs_device(int n, int nrhs, const double* d_a, int lda, const int* d_ipiv, double* d_b, int ldb) {
  return status_of([&] {
    Runtime& r = rt();
    if (n <= 0 || nrhs <= 0) return 0;
    if (nrhs > 16) {
      note("error: bgpu_dgetrs_device takes at most 16 right-hand sides per call");
      return 1;
    }
    DevBuf perm;
    perm.ensure(sizeof(int) * n, "permutation");
    r.ensure_trsv(n);
    ck(cudaEventRecord(r.ev[6], r.stream), "event");
    ck(lu_perm_from_ipiv(d_ipiv, n, perm.as<int>(), r.stream), "permutation");
    ck(getrs64(d_a, lda, n, perm.as<int>(), d_b, ldb, nrhs, r.trsv_scratch.p, r.status.as<int>(), r.stream),
       "solve");
    ck(cudaEventRecord(r.ev[7], r.stream), "event");
    r.check_status("dgetrs");
    r.ms[3] = r.elapsed(6, 7);
    return 0;
  });
}

int bgpu_dgemm_minus_device(int m, int n, int k, const double* d_a, int lda, const double* d_b, int ldb, double* d_c,
                            int ldc) {
  return status_of([&] {
    Runtime& r = rt();
    if ((lda & 1) || (ldb & 1) || ((uintptr_t)d_a & 15) || ((uintptr_t)d_b & 15)) {
      note("error: bgpu_dgemm_minus_device needs even leading dimensions and 16-byte aligned A and B");
      return 1;
    }
    ck(cudaEventRecord(r.ev[6], r.stream), "event");
    ck(dgemm_nn_minus(m, n, k, d_a, lda, d_b, ldb, d_c, ldc, r.stream), "dgemm");
    ck(cudaEventRecord(r.ev[7], r.stream), "event");
    r.sync("dgemm");
    r.ms[3] = r.elapsed(6, 7);
    return 0;
  });
}

unsigned long long bgpu_launch_count(void) { return g_launches; }

int bgpu_kernel_stats(int kernel, int enable, int* launches, double* ms, double* work) {
  return status_of([&] {
    if (kernel < 0 || kernel >= kTimedKernels) {
      note("error: unknown kernel id %d", kernel);
      return 1;
    }
    int l = 0;
    double t = 0, w = 0;
    KernelTimer& kt = kernel_timer(kernel);
    kt.read(&l, &t, &w);
    if (launches) *launches = l;
    if (ms) *ms = t;
    if (work) *work = w;
    kt.enable(enable != 0);
    return 0;
  });
}

int bgpu_gemm_bf16_minus_device(int m, int n, int k, const float* d_a, int lda, const float* d_b, int ldb, float* d_c,
                                int ldc) {
  return status_of([&] {
    Runtime& r = rt();
    if (m <= 0 || n <= 0 || k <= 0) return 0;
    const long lt = ((long)k + 63) / 64 * 64;
    DevBuf at, bt;
    at.ensure((size_t)m * lt * 2, "BF16 A");
    bt.ensure((size_t)n * lt * 2, "BF16 B");
    ck(cudaEventRecord(r.ev[6], r.stream), "event");
    ck(cast_transpose_bf16(d_a, lda, m, k, at.p, lt, r.stream), "cast A");
    ck(cast_bf16(d_b, ldb, k, n, bt.p, lt, r.stream), "cast B");
    KernelTimer& kt = kernel_timer(BGPU_KERNEL_TC_GEMM);
    kt.begin(r.stream);
    ck(gemm_bf16_tc_minus(m, n, k, at.p, lt, bt.p, lt, d_c, ldc, r.status.as<int>(), r.stream), "tensor-core GEMM");
    kt.end(r.stream, 2.0 * m * n * (double)k);
    ck(cudaEventRecord(r.ev[7], r.stream), "event");
    r.check_status("tensor-core GEMM");
    r.ms[3] = r.elapsed(6, 7);
    return 0;
  });
}

int bgpu_set_wait_limit(unsigned spins) {
  return status_of([&] {
    rt();
    ck(set_wait_limit(spins), "wait limit");
    return 0;
  });
}

int bgpu_lu32_leaf_device(int h, float* d_a, int lda, float* d_linv, float* d_uinv) {
  return status_of([&] {
    Runtime& r = rt();
    if (h < 1 || h > 128 || lda < h) {
      note("error: bgpu_lu32_leaf_device: h %d outside 1..128 or lda %d < h", h, lda);
      return 1;
    }
    ck(lu32_leaf(d_a, lda, h, d_linv, d_uinv, r.status.as<int>(), r.stream), "LU leaf");
    r.check_status("LU leaf");
    return 0;
  });
}

int bgpu_trsm_leaf_device(int left, int n, float* d_a, int lda, const float* d_linv, const float* d_uinv, int kd,
                          int p0, int h, int len, void* d_mirror, int ldm) {
  return status_of([&] {
    Runtime& r = rt();
    const bool bad = n < 1 || lda < n || h < 1 || h > 128 || len < 0 || kd < 0 || p0 < 0 || kd % 32 || p0 % 32 ||
                     kd + h > n || p0 + len > n || (d_mirror && ldm < n);
    if (bad) {
      note("error: bgpu_trsm_leaf_device: n %d, lda %d, kd %d, p0 %d, h %d, len %d, ldm %d out of range", n, lda, kd,
           p0, h, len, ldm);
      return 1;
    }
    ck(tc_gemm_prepare(), "tensor-core attributes");
    alignas(64) unsigned char maps[kPanelMaps * kTensorMapBytes];
    if (!tc_panel_maps(d_a, n, lda, d_linv, d_uinv, maps)) {
      note("error: bgpu_trsm_leaf_device: cannot build the tensor maps (lda a multiple of 4, 16-byte aligned buffers)");
      return 1;
    }
    float* X = left ? d_a + kd + (size_t)p0 * lda : d_a + p0 + (size_t)kd * lda;
    void* mir = nullptr;
    alignas(64) unsigned char mmaps[2 * kTensorMapBytes];
    if (d_mirror) {
      auto* m = static_cast<uint16_t*>(d_mirror);
      mir = left ? (void*)(m + kd + (size_t)p0 * ldm) : (void*)(m + (size_t)p0 * ldm + kd);
      if (!tc_mirror_store_maps(d_mirror, d_mirror, n, ldm, mmaps)) {
        note("error: bgpu_trsm_leaf_device: cannot build the mirror's tensor maps (ldm a multiple of 8, aligned)");
        return 1;
      }
    }
    if (left)
      ck(panel_tf32(true, false, maps, kMapDL, kMapK, mmaps, 0, kd, kd, p0, h, len, X, lda, kd, p0, mir, ldm,
                    r.status.as<int>(), r.stream, nullptr),
         "triangular-solve leaf");
    else
      ck(panel_tf32(false, false, maps, kMapDU, kMapMN, mmaps, 0, kd, p0, kd, h, len, X, lda, p0, kd, mir, ldm,
                    r.status.as<int>(), r.stream, nullptr),
         "triangular-solve leaf");
    r.check_status("triangular-solve leaf");
    return 0;
  });
}

int bgpu_trsm_leaf256_device(int left, int n, float* d_a, int lda, const float* d_linv, const float* d_uinv, int kd,
                             int p0, int len, void* d_mirror, int ldm) {
  return status_of([&] {
    Runtime& r = rt();
    const bool bad = n < 1 || lda < n || lda % 4 || len < 1 || kd < 0 || p0 < 0 || kd % 128 || p0 % 32 ||
                     kd + 256 > n || p0 + len > n || (d_mirror && (ldm < n || ldm % 8));
    if (bad) {
      note("error: bgpu_trsm_leaf256_device: n %d, lda %d, kd %d, p0 %d, len %d, ldm %d out of range", n, lda, kd, p0,
           len, ldm);
      return 1;
    }
    ck(tc_gemm_prepare(), "tensor-core attributes");
    const int slots = (n + 127) / 128;
    DevBuf tl, tu;
    tl.ensure((size_t)slots * 65536 * sizeof(float), "256-block inverses (L)");
    tu.ensure((size_t)slots * 65536 * sizeof(float), "256-block inverses (U)");
    alignas(64) unsigned char maps[kPanelMaps * kTensorMapBytes], tmaps[2 * kTensorMapBytes],
        mmaps[2 * kTensorMapBytes];
    if (!tc_panel_maps(d_a, n, lda, d_linv, d_uinv, maps) ||
        !tc_leaf256_maps(tl.as<float>(), tu.as<float>(), slots, tmaps) ||
        (d_mirror && !tc_mirror_store_maps(d_mirror, d_mirror, n, ldm, mmaps))) {
      note("error: bgpu_trsm_leaf256_device: cannot build the tensor maps");
      return 1;
    }
    ck(combine256(d_a, lda, kd, d_linv, d_uinv, tl.as<float>(), tu.as<float>(), r.stream), "256-block inverses");
    float* X = left ? d_a + kd + (size_t)p0 * lda : d_a + p0 + (size_t)kd * lda;
    void* mir = nullptr;
    if (d_mirror) {
      auto* m = static_cast<uint16_t*>(d_mirror);
      mir = left ? (void*)(m + kd + (size_t)p0 * ldm) : (void*)(m + (size_t)p0 * ldm + kd);
    }
    ck(leaf256_tf32(left != 0, maps, tmaps, d_mirror ? mmaps : nullptr, kd / 128, kd, p0, 256, len, X, lda, mir, ldm,
                    r.status.as<int>(), r.stream, nullptr),
       "256-deep triangular-solve leaf");
    r.check_status("256-deep triangular-solve leaf");  // (synchronises before the buffers go)
    return 0;
  });
}

int bgpu_panel_update_device(int n, float* d_a, int lda, int m, int nc, int ar, int ac, int br, int bc, int cr,
                             int cc) {
  return status_of([&] {
    Runtime& r = rt();
    auto in = [&](int r0, int c0, int rows, int cols) { return r0 >= 0 && c0 >= 0 && r0 + rows <= n && c0 + cols <= n; };
    const bool bad = n < 1 || lda < n || m < 1 || nc < 1 || std::min(m, nc) > 256 || ar % 4 || br % 4 || cr % 4 ||
                     !in(ar, ac, m, 128) || !in(br, bc, 128, nc) || !in(cr, cc, m, nc);
    if (bad) {
      note("error: bgpu_panel_update_device: blocks outside the %d x %d matrix, both sides above 256, or a row offset "
           "not a multiple of 4", n, n);
      return 1;
    }
    ck(tc_gemm_prepare(), "tensor-core attributes");
    alignas(64) unsigned char maps[kPanelMaps * kTensorMapBytes];
    // the diagonal-block maps are not used: any aligned buffer stands in for them
    if (!tc_panel_maps(d_a, n, lda, d_a, d_a, maps)) {
      note("error: bgpu_panel_update_device: cannot build the tensor maps (lda a multiple of 4, 16-byte aligned)");
      return 1;
    }
    float* C = d_a + cr + (size_t)cc * lda;
    if (m <= nc)
      ck(panel_tf32(true, true, maps, kMapMN, kMapK, nullptr, ar, ac, br, bc, m, nc, C, lda, cr, cc, nullptr, 0,
                    r.status.as<int>(), r.stream, nullptr),
         "panel update");
    else
      ck(panel_tf32(false, true, maps, kMapK, kMapMN, nullptr, br, bc, ar, ac, nc, m, C, lda, cr, cc, nullptr, 0,
                    r.status.as<int>(), r.stream, nullptr),
         "panel update");
    r.check_status("panel update");
    return 0;
  });
}

static int assemble_device(bool fast, int r0, int r1, int c0, int c1, double* d_out, int ldo) {
  return status_of([&] {
    Solver& s = solver();
    Runtime& r = rt();
    if (r0 < 0 || c0 < 0 || r1 > s.n || c1 > s.n || ldo < 3 * (r1 - r0)) {
      note("error: bgpu_assemble_device: range outside the mesh or ldo too small");
      return 1;
    }
    DevDeflation none;
    ck(cudaEventRecord(r.ev[2], r.stream), "event");
    if (fast)
      ck(launch_assemble_fast(s.mesh(), r0, r1, c0, c1, d_out, ldo, none, nullptr, 0, r.stream), "assembly");
    else
      ck(launch_assemble(s.mesh(), r0, r1, c0, c1, d_out, ldo, none, nullptr, 0, r.stream), "assembly");
    ck(cudaEventRecord(r.ev[3], r.stream), "event");
    r.sync("assembly");
    r.ms[1] = r.elapsed(2, 3);
    return 0;
  });
}

int bgpu_assemble_device(int r0, int r1, int c0, int c1, double* d_out, int ldo) {
  return assemble_device(false, r0, r1, c0, c1, d_out, ldo);
}

int bgpu_assemble_device_mixed(int r0, int r1, int c0, int c1, double* d_out, int ldo) {
  return assemble_device(true, r0, r1, c0, c1, d_out, ldo);
}

}  // extern "C"
