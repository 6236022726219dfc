"""best_hydro_b200: BEST's dense boundary-element hot path on one B200.

The product is the shared library ``lib/libbestgpu.so`` (CUDA kernels for sm_100a behind the C ABI
of ``include/best_hmatrix.h`` and ``include/best_gpu.h``).  This module is a thin ctypes mirror of
that interface for Python callers (tests, benchmarks): it loads the in-tree library and raises if it
is missing; there is no Python or CPU implementation of any stage behind it.

    from best_hydro_b200 import BhmSolver
    s = BhmSolver()
    s.create(v1, v2, v3, area, afac, cg)     # bhm_create
    x = s.incenters()                         # bhm_incenters
    dm = s.diag_mean()                        # bhm_diag_mean
    s.build(eps, direct, ndef, gdef, comp, xmu)   # bhm_build
    b = s.solve(b)                            # bhm_solve
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "lib", "libbestgpu.so")

BGPU_FP64 = 0
BGPU_MIXED = 1
BGPU_HMATRIX = 2

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None

# name -> (restype, argtypes), as declared in include/best_hmatrix.h and include/best_gpu.h
_SIGS = {
    "bhm_available": (ctypes.c_int, []),
    "bhm_create": (ctypes.c_int, [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "bhm_incenters": (None, [_dp]),
    "bhm_entries": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]),
    "bhm_diag_mean": (ctypes.c_double, []),
    "bhm_build": (ctypes.c_int, [ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _ip, _dp,
                                 ctypes.c_int, ctypes.c_int]),
    "bhm_solve": (ctypes.c_int, [ctypes.c_int, _dp]),
    "bhm_log_line": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "bhm_destroy": (None, []),
    "bgpu_set_precision": (ctypes.c_int, [ctypes.c_int]),
    "bgpu_precision": (ctypes.c_int, []),
    "bgpu_set_refinement": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "bgpu_timings": (ctypes.c_int, [_dp, ctypes.c_int]),
    "bgpu_stream": (ctypes.c_void_p, []),
    "bgpu_solve_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "bgpu_dgetrf_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, _ip]),
    "bgpu_dgetrs_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_int]),
    "bgpu_dgetrs_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "bgpu_dgemm_minus_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "bgpu_gemm_bf16_minus_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                   ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                   ctypes.c_int]),
    "bgpu_assemble_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_int]),
    "bgpu_assemble_device_mixed": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_void_p, ctypes.c_int]),
    "bgpu_series_create": (ctypes.c_int, [ctypes.c_int, _ip, _dp, _dp, _dp, _dp, _dp, ctypes.c_double]),
    "bgpu_series_incenters": (ctypes.c_int, [_dp]),
    "bgpu_series_diag_mean": (ctypes.c_int, [_dp]),
    "bgpu_series_build": (ctypes.c_int, [_ip, _dp, _ip, _dp, ctypes.c_int]),
    "bgpu_series_solve": (ctypes.c_int, [ctypes.c_int, _dp]),
    "bgpu_series_timings": (ctypes.c_int, [_dp, ctypes.c_int]),
    "bgpu_series_destroy": (None, []),
    "bgpu_series_set_precision": (ctypes.c_int, [ctypes.c_int]),
    "bgpu_autotune_table": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "bgpu_best_gradient": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp]),
    "bgpu_set_wait_limit": (ctypes.c_int, [ctypes.c_uint]),
    "bgpu_lu32_leaf_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p]),
    "bgpu_trsm_leaf_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_int]),
    "bgpu_panel_update_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p] + [ctypes.c_int] * 9),
    "bgpu_trsm_leaf256_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "bgpu_create_from_triangles": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                  _dp, _ip]),
    "bgpu_build_prepared": (ctypes.c_int, [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bgpu_prepared_arrays": (ctypes.c_int, [_dp, _dp, _dp, _dp, _ip, _dp, _dp]),
    "bgpu_launch_count": (ctypes.c_ulonglong, []),
    "bgpu_kernel_stats": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _ip, _dp, _dp]),
    "bgpu_hmatrix_set_options": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "bgpu_hmatrix_stats": (ctypes.c_int, [_dp, ctypes.c_int]),
    "bgpu_hmatrix_matvec_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_int]),
    "bgpu_hmatrix_plan": (ctypes.c_int, [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, _ip, _ip]),
    # include/best_driver.h: BEST's host side around the seam
    "bgpu_best_setup": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, _dp,
                                       _dp, _ip, _ip, _ip, _ip]),
    "bgpu_best_deflation": (ctypes.c_int, [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, _ip, ctypes.c_double, _dp,
                                           _dp]),
    "bgpu_best_rhs6": (None, [ctypes.c_int, _dp, _dp]),
    "bgpu_best_strain5": (None, [ctypes.c_int, _dp, _dp]),
    "bgpu_best_difco": (ctypes.c_int, [ctypes.c_int, _dp, _dp, ctypes.c_double, _dp, _dp]),
    "bgpu_best_visco": (ctypes.c_int, [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp]),
    "bgpu_best_traces": (None, [_dp, _dp]),
    "bgpu_best_extrapolate": (ctypes.c_double, [ctypes.c_int, _ip, _dp, _dp]),
    "bgpu_best_run": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_int, _dp]),
}


class BestGpuError(RuntimeError):
    pass


def lib():
    """The loaded libbestgpu (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise BestGpuError(f"libbestgpu is not built ({LIBPATH}); run python -m best_hydro_b200.build")
        L = ctypes.CDLL(LIBPATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def log_lines():
    """Drains the library's message queue (bhm_log_line)."""
    L = lib()
    out = []
    buf = ctypes.create_string_buffer(1024)
    while True:
        k = L.bhm_log_line(buf, 1024)
        if k < 0:
            return out
        out.append(buf.raw[:k].decode(errors="replace"))


def _check(rc, what):
    if rc != 0:
        raise BestGpuError(f"{what} failed: " + " | ".join(log_lines()))


def _p(a):
    return a.ctypes.data_as(_dp)


def timings():
    """Stage times (ms) of the last calls: dict of bgpu_timings."""
    v = np.zeros(7)
    lib().bgpu_timings(_p(v), 7)
    keys = ("create", "assemble", "factor", "solve", "build", "refine_iters", "relres")
    return dict(zip(keys, v.tolist()))


class BhmSolver:
    """The nine-function seam of BEST (include/best_hmatrix.h), one solver per process."""

    def __init__(self):
        self.L = lib()
        self.n = 0

    @staticmethod
    def available():
        return bool(lib().bhm_available())

    def create(self, v1, v2, v3, area, afac, cg=1.0):
        """v1, v2, v3: BEST's n x 3 column-major arrays flattened (v[c*n+i]); area corrected."""
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (v1, v2, v3, area)]
        n = self._keep[3].size
        _check(self.L.bhm_create(n, *(_p(a) for a in self._keep), float(afac), float(cg), 0), "bhm_create")
        self.n = n

    def incenters(self):
        x = np.empty(3 * self.n)
        self.L.bhm_incenters(_p(x))
        return x

    def entries(self, i0, m, j0, nc):
        a = np.zeros((m, nc), dtype=np.float64, order="F")
        self.L.bhm_entries(i0, m, j0, nc, a.ctypes.data_as(_dp), m)
        return a

    def diag_mean(self):
        return float(self.L.bhm_diag_mean())

    def build(self, eps=1e-4, direct=1, ndef=1, gdef=None, comp=None, xmu=None, single=0, nrhs=6):
        gdef = np.ascontiguousarray(gdef, dtype=np.float64)
        comp = np.ascontiguousarray(comp if comp is not None else np.ones(self.n), dtype=np.int32)
        xmu = np.ascontiguousarray(xmu, dtype=np.float64)
        _check(self.L.bhm_build(float(eps), int(direct), 0.1, int(ndef), _p(gdef), comp.ctypes.data_as(_ip), _p(xmu),
                                int(single), int(nrhs)), "bhm_build")

    def solve(self, b):
        b = np.array(b, dtype=np.float64, order="F", copy=True)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        _check(self.L.bhm_solve(nrhs, _p(b)), "bhm_solve")
        return b

    def solve_device(self, d_b, nrhs, ldb):
        _check(self.L.bgpu_solve_device(int(nrhs), ctypes.c_void_p(d_b), int(ldb)), "bgpu_solve_device")

    def gradient(self, iarea=1, truearea=0.0, wm=0.0):
        """bgpu_best_gradient: (values [D_t, D_r, [eta] or CHI'], gradients (3 results, N triangles,
        3 corners, 3 coordinates)) with respect to the corners as read (before the centroid shift)."""
        n = self.n
        vals = np.zeros(3)
        g = np.zeros(27 * n)
        _check(self.L.bgpu_best_gradient(int(iarea), float(truearea or 0.0), float(wm), _p(vals), _p(g)),
               "bgpu_best_gradient")
        return vals, g.reshape(3, 3, 3, n).transpose(0, 3, 1, 2).copy()

    def create_from_triangles(self, tri, iarea=1, truearea=None, cg=1.0):
        """bgpu_create_from_triangles: BEST's set-up and COMPON on the GPU from the triangles as read
        (n x 9).  Returns (info {afac, totarea, centroid}, counts {ncomp, nopen, ndef})."""
        tri = np.ascontiguousarray(tri, dtype=np.float64).reshape(-1, 9)
        n = tri.shape[0]
        info = np.zeros(5)
        counts = np.zeros(3, dtype=np.int32)
        _check(self.L.bgpu_create_from_triangles(n, _p(tri), int(iarea), float(truearea or 0.0), float(cg), _p(info),
                                                 counts.ctypes.data_as(_ip)), "bgpu_create_from_triangles")
        self.n = n
        return (dict(afac=float(info[0]), totarea=float(info[1]), centroid=info[2:5].copy()),
                dict(ncomp=int(counts[0]), nopen=int(counts[1]), ndef=int(counts[2])))

    def build_prepared(self, eps=1e-4, direct=1, single=0, nrhs=6):
        """bgpu_build_prepared: the deflation on the GPU, then the build."""
        _check(self.L.bgpu_build_prepared(float(eps), int(direct), int(single), int(nrhs)), "bgpu_build_prepared")

    def prepared_arrays(self, ndef):
        """bgpu_prepared_arrays: (v1, v2, v3, area, icomp, xmu, gdef) of the device set-up."""
        n = self.n
        v = [np.zeros(3 * n) for _ in range(3)]
        area = np.zeros(n)
        icomp = np.zeros(n, dtype=np.int32)
        xmu = np.zeros(3 * n)
        gdef = np.zeros(max(1, ndef))
        _check(self.L.bgpu_prepared_arrays(_p(v[0]), _p(v[1]), _p(v[2]), _p(area), icomp.ctypes.data_as(_ip), _p(xmu),
                                           _p(gdef)), "bgpu_prepared_arrays")
        return v[0], v[1], v[2], area, icomp, xmu, gdef[:max(1, ndef)]

    def destroy(self):
        self.L.bhm_destroy()
        self.n = 0


class Setup:
    """BEST's arrays after its set-up (best/best.f:261-337), from the C++ host driver."""

    def __init__(self, tri, iarea=1, truearea=None):
        tri = np.ascontiguousarray(tri, dtype=np.float64)
        n = tri.shape[0]
        self.n = n
        self.v1, self.v2, self.v3 = (np.empty(3 * n) for _ in range(3))
        self.area = np.empty(n)
        self.icomp = np.empty(n, dtype=np.int32)
        a, t = ctypes.c_double(), ctypes.c_double()
        cen = np.empty(3)
        nc, no, nd = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        rc = lib().bgpu_best_setup(n, _p(tri), int(iarea), float(truearea or 0.0), _p(self.v1), _p(self.v2),
                                   _p(self.v3), _p(self.area), ctypes.byref(a), ctypes.byref(t), _p(cen),
                                   self.icomp.ctypes.data_as(_ip), ctypes.byref(nc), ctypes.byref(no),
                                   ctypes.byref(nd))
        if rc:
            raise BestGpuError("bgpu_best_setup failed")
        self.afac, self.totarea, self.centroid = a.value, t.value, cen
        self.ncomp, self.nopen, self.ndef = nc.value, no.value, nd.value

    def deflation(self, diagm):
        xmu = np.empty(3 * self.n)
        gdef = np.empty(max(1, self.ndef))
        lib().bgpu_best_deflation(self.n, _p(self.v1), _p(self.v2), _p(self.v3), _p(self.area), self.ndef,
                                  self.icomp.ctypes.data_as(_ip), float(diagm), _p(xmu), _p(gdef))
        return xmu, gdef


def rhs6(x):
    n = x.size // 3
    b = np.empty((3 * n, 6), order="F")
    lib().bgpu_best_rhs6(n, _p(np.ascontiguousarray(x)), b.ctypes.data_as(_dp))
    return b


def strain5(x):
    n = x.size // 3
    v = np.empty((3 * n, 5), order="F")
    lib().bgpu_best_strain5(n, _p(np.ascontiguousarray(x)), v.ctypes.data_as(_dp))
    return v


TENSOR_KEYS = (("Dtt", 0, 9), ("Dtr", 9, 9), ("Drr", 18, 9), ("urc", 27, 3), ("udr", 30, 3), ("Ktt", 33, 9),
               ("KrtCR", 42, 9), ("KrrCR", 51, 9))


def _unpack(out):
    return {k: (out[o:o + m].reshape(3, 3).copy() if m == 9 else out[o:o + m].copy()) for k, o, m in TENSOR_KEYS}


def difco(x, area, b6, cg=1.0):
    """best/difco.f on the six solutions: dict of Dtt, Dtr, Drr, urc, udr, Ktt, KrtCR, KrrCR."""
    n = area.size
    out = np.empty(60)
    b6 = np.asfortranarray(b6, dtype=np.float64)
    lib().bgpu_best_difco(n, _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(area)), float(cg),
                          b6.ctypes.data_as(_dp), _p(out))
    return _unpack(out)


def visco(x, area, v5, b6, icov=0, cg=1.0):
    """best/visco.f: (CHI', (Dx, Dy, Dz))."""
    n = area.size
    out = np.empty(4)
    v5 = np.asfortranarray(v5, dtype=np.float64)
    b6 = np.asfortranarray(b6, dtype=np.float64)
    lib().bgpu_best_visco(n, _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(area)), float(cg), int(icov),
                          v5.ctypes.data_as(_dp), b6.ctypes.data_as(_dp), _p(out))
    return float(out[0]), (float(out[1]), float(out[2]), float(out[3]))


def traces(t):
    """best/output.f:96-130 from difco's tensors: dict trace_dtt, trace_drr, DTRANS, DR."""
    buf = np.zeros(60)
    for k, o, m in TENSOR_KEYS:
        buf[o:o + m] = np.asarray(t[k]).ravel()
    out = np.empty(4)
    lib().bgpu_best_traces(_p(buf), _p(out))
    return dict(trace_dtt=float(out[0]), trace_drr=float(out[1]), DTRANS=float(out[2]), DR=float(out[3]))


def best_run(path, iarea=1, cg_zero=0, ivisco=0, icov=0, wm=0.0, precision=-1):
    """The whole BEST program on the GPU (writes <path><flags>.be and .log); returns a dict."""
    out = np.zeros(68)
    _check(lib().bgpu_best_run(str(path).encode(), int(iarea), int(cg_zero), int(ivisco), int(icov), float(wm),
                               int(precision), _p(out)), "bgpu_best_run")
    d = _unpack(out[:60])
    d.update(chiprime=out[60], dvisc=tuple(out[61:64]), DTRANS=out[64], DR=out[65], CHI=out[66], ETA=out[67])
    return d


BGPU_KERNEL_LU_GEMM64 = 0
BGPU_KERNEL_TC_GEMM = 1


def extrapolate(n, y):
    """bgpu_best_extrapolate: (value at 1/N -> 0, slope) of the least-squares line y = y0 + slope / N."""
    n = np.ascontiguousarray(n, dtype=np.int32)
    y = np.ascontiguousarray(y, dtype=np.float64)
    slope = ctypes.c_double()
    y0 = lib().bgpu_best_extrapolate(int(n.size), n.ctypes.data_as(_ip), _p(y), ctypes.byref(slope))
    return float(y0), slope.value


class Series:
    """A series of meshes solved together (include/best_gpu.h, bgpu_series_*): one assembly launch,
    a batched FP64 LU replayed from one CUDA graph, and per-mesh results equal to single solves."""

    def __init__(self):
        self.L = lib()
        self.n = None

    def create(self, setups, cg=1.0):
        """setups: Setup objects (one per mesh, BEST's set-up already applied)."""
        self.setups = list(setups)
        self.n = np.array([st.n for st in self.setups], dtype=np.int32)
        v1 = np.concatenate([st.v1 for st in self.setups])
        v2 = np.concatenate([st.v2 for st in self.setups])
        v3 = np.concatenate([st.v3 for st in self.setups])
        area = np.concatenate([st.area for st in self.setups])
        afac = np.array([st.afac for st in self.setups], dtype=np.float64)
        _check(self.L.bgpu_series_create(len(self.setups), self.n.ctypes.data_as(_ip), _p(v1), _p(v2), _p(v3),
                                         _p(area), _p(afac), float(cg)), "bgpu_series_create")

    def _split(self, a, per):
        out, o = [], 0
        for k in self.n:
            out.append(a[o:o + per * int(k)])
            o += per * int(k)
        return out

    def incenters(self):
        x = np.empty(3 * int(self.n.sum()))
        _check(self.L.bgpu_series_incenters(_p(x)), "bgpu_series_incenters")
        return self._split(x, 3)

    def diag_means(self):
        dm = np.empty(self.n.size)
        _check(self.L.bgpu_series_diag_mean(_p(dm)), "bgpu_series_diag_mean")
        return dm

    def build(self, deflations, tune=0):
        """deflations: (ndef, gdef, comp, xmu) per mesh."""
        ndef = np.array([d[0] for d in deflations], dtype=np.int32)
        gdef = np.concatenate([np.asarray(d[1], dtype=np.float64)[:max(0, int(d[0]))] for d in deflations])
        comp = np.concatenate([np.asarray(d[2], dtype=np.int32) for d in deflations])
        xmu = np.concatenate([np.asarray(d[3], dtype=np.float64) for d in deflations])
        gdef = np.ascontiguousarray(gdef if gdef.size else np.zeros(1))
        _check(self.L.bgpu_series_build(ndef.ctypes.data_as(_ip), _p(gdef), comp.ctypes.data_as(_ip), _p(xmu),
                                        int(tune)), "bgpu_series_build")

    def solve(self, blocks):
        """blocks: one 3 n_i x nrhs array per mesh (same nrhs); returns the solutions likewise."""
        nrhs = blocks[0].shape[1]
        b = np.concatenate([np.asfortranarray(x, dtype=np.float64).ravel(order="F") for x in blocks])
        _check(self.L.bgpu_series_solve(int(nrhs), _p(b)), "bgpu_series_solve")
        out, o = [], 0
        for k in self.n:
            m = 3 * int(k) * nrhs
            out.append(b[o:o + m].reshape((3 * int(k), nrhs), order="F"))
            o += m
        return out

    def set_precision(self, mode):
        """bgpu_series_set_precision: BGPU_FP64 (batched FP64 LU) or BGPU_MIXED (per-mesh tensor-core
        factorisations side by side, FP64 GMRES-IR) for the next build."""
        _check(self.L.bgpu_series_set_precision(int(mode)), "bgpu_series_set_precision")

    def timings(self):
        v = np.zeros(4)
        self.L.bgpu_series_timings(_p(v), 4)
        return dict(zip(("build", "assemble", "solve", "tune"), v.tolist()))

    def destroy(self):
        self.L.bgpu_series_destroy()


def autotune_table():
    """The DGEMM autotuner's choices (bgpu_autotune_table), one line per size class."""
    k = lib().bgpu_autotune_table(None, 0)
    buf = ctypes.create_string_buffer(k + 1)
    lib().bgpu_autotune_table(buf, k + 1)
    return [ln for ln in buf.value.decode().split("\n") if ln]


def series_run(setups, tune=0, ivisco=1, cg=1.0, precision=None):
    """BEST on every mesh of a series through bgpu_series_*: per mesh D_t, D_r, CHI' (11 right-hand
    sides with ivisco), then their linear extrapolation in 1/N.  precision: None (FP64) or BGPU_MIXED.
    Returns (per-mesh list, extrapolated)."""
    S = Series()
    S.create(setups, cg)
    if precision is not None:
        S.set_precision(precision)
    xs = S.incenters()
    dms = S.diag_means()
    defl = []
    for st, dm in zip(setups, dms):
        xmu, gdef = st.deflation(dm)
        defl.append((st.ndef, gdef, st.icomp, xmu))
    S.build(defl, tune=tune)
    rhs = [np.hstack([rhs6(x), strain5(x)]) if ivisco else rhs6(x) for x in xs]
    sols = S.solve(rhs)
    per = []
    for st, x, B in zip(setups, xs, sols):
        t = difco(x, st.area, B[:, :6], cg)
        tr = traces(t)
        d = dict(N=st.n, D_t=tr["DTRANS"], D_r=tr["DR"], tensors=t, solution=B)
        if ivisco:
            d["chiprime"], _ = visco(x, st.area, B[:, 6:], B[:, :6], 0, cg)
        per.append(d)
    n = [d["N"] for d in per]
    ext = {k: extrapolate(n, [d[k] for d in per])[0] for k in (("D_t", "D_r", "chiprime") if ivisco else ("D_t", "D_r"))}
    timings = S.timings()
    S.destroy()
    return per, ext, timings


def kernel_stats(kernel=BGPU_KERNEL_LU_GEMM64, enable=1):
    """(launches, ms, flops) recorded since the last call; then recording on/off."""
    l, t, w = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
    _check(lib().bgpu_kernel_stats(int(kernel), int(enable), ctypes.byref(l), ctypes.byref(t), ctypes.byref(w)),
           "bgpu_kernel_stats")
    return l.value, t.value, w.value


def launch_count():
    """Kernel launches the library has issued (bgpu_launch_count)."""
    return int(lib().bgpu_launch_count())


def set_refinement(max_restarts=8, krylov=10):
    _check(lib().bgpu_set_refinement(int(max_restarts), int(krylov)), "bgpu_set_refinement")


def set_precision(mode):
    _check(lib().bgpu_set_precision(int(mode)), "bgpu_set_precision")


HMATRIX_STATS = ("n", "leaves", "dense_blocks", "lowrank_blocks", "dense_entries", "lowrank_entries", "mean_rank",
                 "max_rank", "capped_blocks", "fill_ms", "aca_ms", "precond_ms", "gmres_steps", "relres",
                 "device_bytes")


def hmatrix_set_options(leaf=128, eta=2.0, kmax=90):
    """bgpu_hmatrix_set_options: leaf size, admissibility and rank cap of later H-matrix builds."""
    _check(lib().bgpu_hmatrix_set_options(int(leaf), float(eta), int(kmax)), "bgpu_hmatrix_set_options")


def hmatrix_stats():
    """bgpu_hmatrix_stats as a dict (HMATRIX_STATS)."""
    out = np.zeros(len(HMATRIX_STATS))
    _check(lib().bgpu_hmatrix_stats(_p(out), len(out)), "bgpu_hmatrix_stats")
    return dict(zip(HMATRIX_STATS, out.tolist()))


def hmatrix_matvec_device(nrhs, d_x, ldx, d_y, ldy):
    _check(lib().bgpu_hmatrix_matvec_device(int(nrhs), ctypes.c_void_p(d_x), int(ldx), ctypes.c_void_p(d_y),
                                            int(ldy)), "bgpu_hmatrix_matvec_device")


def hmatrix_plan(x, v1, v2, v3, leaf=128, eta=2.0, kmax=90):
    """bgpu_hmatrix_plan (host only): (perm, {depth, leaves, dense, lowrank, admissible})."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, v1, v2, v3)]
    n = arrs[0].size // 3
    perm = np.zeros(n, dtype=np.int32)
    counts = np.zeros(5, dtype=np.int32)
    _check(lib().bgpu_hmatrix_plan(n, *(_p(a) for a in arrs), int(leaf), float(eta), int(kmax),
                                   perm.ctypes.data_as(_ip), counts.ctypes.data_as(_ip)), "bgpu_hmatrix_plan")
    return perm, dict(zip(("depth", "leaves", "dense", "lowrank", "admissible"), counts.tolist()))


def dgetrf_device(n, d_a, lda, d_ipiv):
    """dgetrf on device pointers; returns info."""
    info = ctypes.c_int(0)
    _check(lib().bgpu_dgetrf_device(int(n), ctypes.c_void_p(d_a), int(lda), ctypes.c_void_p(d_ipiv),
                                    ctypes.byref(info)), "bgpu_dgetrf_device")
    return info.value


def dgetrs_device(n, nrhs, d_a, lda, d_ipiv, d_b, ldb):
    _check(lib().bgpu_dgetrs_device(int(n), int(nrhs), ctypes.c_void_p(d_a), int(lda), ctypes.c_void_p(d_ipiv),
                                    ctypes.c_void_p(d_b), int(ldb)), "bgpu_dgetrs_device")


def dgetrs_noalloc(n, nrhs, d_a, lda, d_ipiv, d_b, ldb, stream=0):
    """bgpu_dgetrs_noalloc: the solve without device allocations (see include/best_gpu.h)."""
    _check(lib().bgpu_dgetrs_noalloc(int(n), int(nrhs), ctypes.c_void_p(d_a), int(lda), ctypes.c_void_p(d_ipiv),
                                     ctypes.c_void_p(d_b), int(ldb), ctypes.c_void_p(stream)), "bgpu_dgetrs_noalloc")


def lu32_leaf_device(h, d_a, lda, d_linv, d_uinv):
    """bgpu_lu32_leaf_device: the mixed LU's 128 x 128 diagonal leaf (see include/best_gpu.h)."""
    _check(lib().bgpu_lu32_leaf_device(int(h), ctypes.c_void_p(d_a), int(lda), ctypes.c_void_p(d_linv),
                                       ctypes.c_void_p(d_uinv)), "bgpu_lu32_leaf_device")


def trsm_leaf_device(left, n, d_a, lda, d_linv, d_uinv, kd, p0, h, length, d_mirror=None, ldm=0):
    """bgpu_trsm_leaf_device: the mixed LU's triangular-solve leaf on the tensor cores (see
    include/best_gpu.h)."""
    _check(lib().bgpu_trsm_leaf_device(int(bool(left)), int(n), ctypes.c_void_p(d_a), int(lda), ctypes.c_void_p(d_linv),
                                       ctypes.c_void_p(d_uinv), int(kd), int(p0), int(h), int(length),
                                       ctypes.c_void_p(d_mirror) if d_mirror else None, int(ldm)),
           "bgpu_trsm_leaf_device")


def trsm_leaf256_device(left, n, d_a, lda, d_linv, d_uinv, kd, p0, length, d_mirror=None, ldm=0):
    """bgpu_trsm_leaf256_device: the mixed LU's 256-deep triangular-solve leaf (see include/best_gpu.h)."""
    _check(lib().bgpu_trsm_leaf256_device(int(bool(left)), int(n), ctypes.c_void_p(d_a), int(lda),
                                          ctypes.c_void_p(d_linv), ctypes.c_void_p(d_uinv), int(kd), int(p0),
                                          int(length), ctypes.c_void_p(d_mirror) if d_mirror else None, int(ldm)),
           "bgpu_trsm_leaf256_device")


def panel_update_device(n, d_a, lda, m, nc, ar, ac, br, bc, cr, cc):
    """bgpu_panel_update_device: the mixed LU's K = 128 update on the tensor cores (see
    include/best_gpu.h)."""
    _check(lib().bgpu_panel_update_device(int(n), ctypes.c_void_p(d_a), int(lda), int(m), int(nc), int(ar), int(ac),
                                          int(br), int(bc), int(cr), int(cc)), "bgpu_panel_update_device")


def dgemm_minus_device(m, n, k, d_a, lda, d_b, ldb, d_c, ldc):
    _check(lib().bgpu_dgemm_minus_device(int(m), int(n), int(k), ctypes.c_void_p(d_a), int(lda), ctypes.c_void_p(d_b),
                                         int(ldb), ctypes.c_void_p(d_c), int(ldc)), "bgpu_dgemm_minus_device")


def gemm_bf16_minus_device(m, n, k, d_a, lda, d_b, ldb, d_c, ldc):
    _check(lib().bgpu_gemm_bf16_minus_device(int(m), int(n), int(k), ctypes.c_void_p(d_a), int(lda),
                                             ctypes.c_void_p(d_b), int(ldb), ctypes.c_void_p(d_c), int(ldc)),
           "bgpu_gemm_bf16_minus_device")


def assemble_device(r0, r1, c0, c1, d_out, ldo, mixed=False):
    """GR block (before deflation) into device memory; mixed=True: the mixed path's assembly."""
    fn = lib().bgpu_assemble_device_mixed if mixed else lib().bgpu_assemble_device
    _check(fn(int(r0), int(r1), int(c0), int(c1), ctypes.c_void_p(d_out), int(ldo)), "bgpu_assemble_device")
