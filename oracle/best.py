"""ORACLE (test infrastructure only): a CPU restatement of BEST's dense path.

This module is the oracle for the CUDA path.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it; the product never does.

It restates, in numpy, the reference's driver arithmetic around the hot path, and calls the C
restatement of the assembly (``oracle/tgetgr.c`` -> ``lib/liborc.so``) or the reference's own
C++ assembly (``hmatrix/src/kernel.cpp`` -> ``_ref/libbestref.so``) for GR.  The LU and solve are
LAPACK ``dgetrf``/``dgetrs`` (scipy's OpenBLAS), the same third-party routines BEST calls
(best/best.f:444, best/besolve.f90:133).

Followed (file:line in the reference):
  read/centroid/areas/AFAC   best/best.f:189-221, :261-283, :287-298, :304-315
  COMPON, DEFGAM             best/compon.f90:19-116, :185-197
  deflation                  best/best.f:384-426
  DIFCO                      best/difco.f:28-401
  MATIN3 (LUDCMP3/LUBKSB3)   best/matin3.f:1-118
  VISCO, STRAIN              best/visco.f:21-243
  JACOBI                     best/jacobi.f:1-96
  OUTPUT units and traces    best/output.f:16-29, :96-171

Fortran semantics kept: every REAL is FP64; sums over triangles are sequential (``_seqsum``
accumulates left to right, as the DO loops do); expressions keep the Fortran order.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)


def _ptr(a):
    return a.ctypes.data_as(_dp)


def lib():
    """The C restatement of TGETGR/triangleint (built by oracle/Makefile)."""
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "lib", "liborc.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        L = ctypes.CDLL(path)
        L.orc_self_blocks.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
        L.orc_gr_block.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, _dp, _dp,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_long]
        L.orc_diag_mean.argtypes = [ctypes.c_int, _dp]
        L.orc_diag_mean.restype = ctypes.c_double
        L.orc_deflate.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _ip, _dp, _dp, ctypes.c_long]
        L.orc_ulp_hist.argtypes = [ctypes.c_long, _dp, _dp, _llp, ctypes.c_int]
        L.orc_ulp_hist.restype = ctypes.c_longlong
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own kernel.cpp behind a C shim (oracle/_ref/libbestref.so), or None."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libbestref.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        L.ref_create.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double]
        L.ref_incenters.argtypes = [_dp]
        L.ref_fill.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_long]
        L.ref_diag_mean.restype = ctypes.c_double
        _REF = L
    return _REF


def _seqsum(v):
    """Left-to-right sum, as a Fortran DO loop accumulates (0.0 + v1 + v2 + ...).  Complex input
    (the complex-step reference gradient, gradref.py) is summed the same way."""
    v = np.asarray(v)
    if not np.iscomplexobj(v):
        v = v.astype(np.float64, copy=False)
    if v.size == 0:
        return 0.0
    r = np.add.accumulate(np.concatenate([[0.0], v]))[-1]
    return complex(r) if np.iscomplexobj(r) else float(r)


def _re(z):
    """The real part (pivoting and zero tests of complex-step runs follow the real computation)."""
    return z.real if isinstance(z, (complex, np.complexfloating)) else z


# ----------------------------------------------------------------------------------------------
# Input and set-up (best.f)
# ----------------------------------------------------------------------------------------------

def read_mesh(path):
    """best.f:189-221: header NAR [TRUEAREA TRUEVOL], then 9 reals per triangle.
    Returns (tri (nar, 9), truearea or None, truevol or None)."""
    with open(path) as f:
        head = f.readline().split()
        nar = int(float(head[0]))
        ta = float(head[1]) if len(head) > 1 else None
        tv = float(head[2]) if len(head) > 2 else None
        data = np.loadtxt(f, dtype=np.float64, max_rows=nar).reshape(nar, 9)
    return data, ta, tv


@dataclass
class Setup:
    n: int
    v1: np.ndarray  # (n, 3) C-order rows; .T.copy() gives BEST's column-major V1(NAR,3)
    v2: np.ndarray
    v3: np.ndarray
    area: np.ndarray  # corrected areas
    afac: float
    totarea: float
    centroid: tuple
    icomp: np.ndarray = field(default=None)
    ncomp: int = 1
    nopen: int = 0
    ndef: int = 1

    def colmajor(self):
        """V1, V2, V3 as BEST holds them: n x 3 column-major, flattened (v[c*n + i])."""
        return (np.ascontiguousarray(self.v1.T).ravel(), np.ascontiguousarray(self.v2.T).ravel(),
                np.ascontiguousarray(self.v3.T).ravel())


def setup(tri, iarea, truearea):
    """best.f:261-315: centroid of triangle centroids subtracted, areas, area correction."""
    tri = np.asarray(tri, dtype=np.float64)
    n = tri.shape[0]
    v1 = tri[:, 0:3].copy()
    v2 = tri[:, 3:6].copy()
    v3 = tri[:, 6:9].copy()
    # cx = cx + (v1+v2+v3)/3 sequentially, then / nar (best.f:261-272)
    cen = []
    for c in range(3):
        cen.append(_seqsum((v1[:, c] + v2[:, c] + v3[:, c]) / 3.0) / n)
    for c in range(3):
        v1[:, c] = v1[:, c] - cen[c]
        v2[:, c] = v2[:, c] - cen[c]
        v3[:, c] = v3[:, c] - cen[c]
    e21 = v2 - v1
    e31 = v3 - v1
    cx_ = e31[:, 1] * e21[:, 2] - e31[:, 2] * e21[:, 1]
    cy_ = e31[:, 2] * e21[:, 0] - e31[:, 0] * e21[:, 2]
    cz_ = e31[:, 0] * e21[:, 1] - e31[:, 1] * e21[:, 0]
    area = np.sqrt(cx_ * cx_ + cy_ * cy_ + cz_ * cz_) * 0.5
    totarea = _seqsum(area)
    if iarea:
        afac = truearea / totarea
        area = afac * area
    else:
        afac = 1.0
    s = Setup(n=n, v1=v1, v2=v2, v3=v3, area=area, afac=afac, totarea=totarea, centroid=tuple(cen))
    compon(s)
    return s


def compon(s: Setup):
    """compon.f90:19-116: surfaces of triangles sharing a vertex (exact coordinates), numbered in
    the order of their first triangles; NOPEN = edges not shared by exactly two triangles.
    best.f:323-337: NDEF = NCOMP for a closed triangulation, else 1 (all ICOMP = 1)."""
    n = s.n
    corners = np.stack([s.v1, s.v2, s.v3], axis=1).reshape(3 * n, 3)  # k = 3*t + c
    _, vid = np.unique(corners, axis=0, return_inverse=True)
    vid = vid.ravel()
    root = list(range(n))

    def find(i):
        p = i
        while root[p] != p:
            p = root[p]
        while root[i] != p:
            root[i], i = p, root[i]
        return p

    order = np.argsort(vid, kind="stable")
    for j in range(1, 3 * n):
        a, b = order[j], order[j - 1]
        if vid[a] == vid[b]:
            ra, rb = find(a // 3), find(b // 3)
            if ra != rb:
                root[max(ra, rb)] = min(ra, rb)
    lab = {}
    icomp = np.zeros(n, dtype=np.int32)
    for t in range(n):
        r = find(t)
        if r not in lab:
            lab[r] = len(lab) + 1
        icomp[t] = lab[r]
    ncomp = len(lab)
    tv = vid.reshape(n, 3)
    ea = np.concatenate([tv[:, 0], tv[:, 1], tv[:, 2]])
    eb = np.concatenate([tv[:, 1], tv[:, 2], tv[:, 0]])
    edges = np.stack([np.minimum(ea, eb), np.maximum(ea, eb)], axis=1)
    _, counts = np.unique(edges, axis=0, return_counts=True)
    nopen = int(np.count_nonzero(counts != 2))
    s.ncomp, s.nopen = ncomp, nopen
    if nopen > 0:
        s.ndef, s.icomp = 1, np.ones(n, dtype=np.int32)
    else:
        s.ndef, s.icomp = ncomp, icomp
    return s


def deflation_vectors(s: Setup, diagm):
    """best.f:384-404 (XMU = area * unit normal, GDEF = DIAGM/|XMU|^2) and DEFGAM
    (compon.f90:185-197) for NDEF > 1.  Returns (xmu (3n,), gdef (ndef,))."""
    e21 = s.v2 - s.v1
    e31 = s.v3 - s.v1
    xnx = e31[:, 1] * e21[:, 2] - e31[:, 2] * e21[:, 1]
    xny = e31[:, 2] * e21[:, 0] - e31[:, 0] * e21[:, 2]
    xnz = e31[:, 0] * e21[:, 1] - e31[:, 1] * e21[:, 0]
    xnl = np.sqrt(xnx * xnx + xny * xny + xnz * xnz)
    xmu = np.empty(3 * s.n)
    xmu[0::3] = s.area * xnx / xnl
    xmu[1::3] = s.area * xny / xnl
    xmu[2::3] = s.area * xnz / xnl
    sq = xmu[0::3] * xmu[0::3] + xmu[1::3] * xmu[1::3] + xmu[2::3] * xmu[2::3]
    if s.ndef == 1:
        # xmu2 = xmu2 + x^2 + y^2 + z^2, triangle by triangle
        acc = 0.0
        for v in zip(xmu[0::3] ** 2, xmu[1::3] ** 2, xmu[2::3] ** 2):
            acc = acc + v[0] + v[1] + v[2]
        gdef = np.array([diagm / acc])
    else:
        g = np.zeros(s.ndef)
        for t in range(s.n):
            k = s.icomp[t] - 1
            g[k] = g[k] + xmu[3 * t] ** 2 + xmu[3 * t + 1] ** 2 + xmu[3 * t + 2] ** 2
        gdef = diagm / g
    del sq
    return xmu, gdef


# ----------------------------------------------------------------------------------------------
# GR (C restatement, or the reference's kernel.cpp)
# ----------------------------------------------------------------------------------------------

def incenters_and_self(s: Setup, cg=1.0):
    """TGETGR's self loop (tgetgr.f:33-147) via liborc: (x (n,3) column-major flattened, self9)."""
    L = lib()
    v1, v2, v3 = s.colmajor()
    x = np.empty(3 * s.n)
    self9 = np.empty(9 * s.n)
    L.orc_self_blocks(s.n, _ptr(v1), _ptr(v2), _ptr(v3), s.afac, cg, _ptr(x), _ptr(self9))
    return x, self9


def assemble(s: Setup, cg=1.0, rows=None, cols=None):
    """GR before deflation (tgetgr.f), column-major (Fortran-ordered ndarray).  rows/cols: triangle
    ranges (r0, r1), (c0, c1) for a sub-block.  Returns (gr, x, self9)."""
    L = lib()
    v1, v2, v3 = s.colmajor()
    x, self9 = incenters_and_self(s, cg)
    r0, r1 = rows if rows else (0, s.n)
    c0, c1 = cols if cols else (0, s.n)
    m, nc = 3 * (r1 - r0), 3 * (c1 - c0)
    gr = np.empty((m, nc), dtype=np.float64, order="F")
    L.orc_gr_block(s.n, _ptr(v1), _ptr(v2), _ptr(v3), _ptr(s.area), cg, _ptr(x), _ptr(self9),
                   r0, r1, c0, c1, gr.ctypes.data_as(_dp), m)
    return gr, x, self9


def assemble_ref(s: Setup, cg=1.0, rows=None, cols=None):
    """The same through the reference's own kernel.cpp (None if _ref is not built)."""
    R = ref_lib()
    if R is None:
        return None
    v1, v2, v3 = s.colmajor()
    R.ref_create(s.n, _ptr(v1), _ptr(v2), _ptr(v3), _ptr(s.area), s.afac, cg)
    x = np.empty(3 * s.n)
    R.ref_incenters(_ptr(x))
    r0, r1 = rows if rows else (0, s.n)
    c0, c1 = cols if cols else (0, s.n)
    m, nc = 3 * (r1 - r0), 3 * (c1 - c0)
    gr = np.empty((m, nc), dtype=np.float64, order="F")
    R.ref_fill(r0, r1, c0, c1, gr.ctypes.data_as(_dp), m)
    dm = R.ref_diag_mean()
    R.ref_destroy()
    return gr, x, dm


# 21-point Gauss-Legendre rule of best/triangleint.f:66-108 (decimal literals)
_GY = (3.1239146898052499e-3, 1.6386580716846853e-2, 3.9950332924799586e-2, 7.3318317708341358e-2,
       0.1157800182621610, 0.1664305979012938, 0.2241905820563901, 0.2878289398962806,
       0.3559893415987995, 0.4272190729195525, 0.5, 0.5727809270804476,
       0.6440106584012005, 0.7121710601037194, 0.7758094179436099, 0.8335694020987062,
       0.8842199817378390, 0.9266816822916586, 0.9600496670752004, 0.9836134192831531,
       0.9968760853101948)
_GW = (1.601722825777433e-2, 3.695378977085249e-2, 5.713442542685720e-2, 7.610011362837930e-2,
       9.344442345603390e-2, 0.1087972991671484, 0.1218314160537285, 0.1322689386333375,
       0.1398873947910731, 0.1445244039899701, 0.1460811336496904, 0.1445244039899701,
       0.1398873947910731, 0.1322689386333375, 0.1218314160537285, 0.1087972991671484,
       9.344442345603390e-2, 7.610011362837930e-2, 5.713442542685720e-2, 3.695378977085249e-2,
       1.601722825777433e-2)


def pair_blocks_ld(s: Setup, x, rows, cols, cg=1.0):
    """The 3x3 pair blocks GR(target rows[k], source cols[k]) (rows != cols) of best/triangleint.f:1-247
    evaluated in numpy's long double (x86 80-bit, 64-bit significand): a reference value about 2^11
    times more precise than any FP64 evaluation, for judging FP64 variants of the quadrature.
    x: incenters as incenters_and_self returns them.  Returns (k, 3, 3) float64."""
    T = np.longdouble
    X = np.asarray(x, dtype=np.float64).reshape(3, -1).T[rows].astype(T)
    P1, P2, P3 = (v[cols].astype(T) for v in (s.v1, s.v2, s.v3))
    area = s.area[cols].astype(T)

    def dot(a, b):
        return a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]

    v21, v31, v32 = P2 - P1, P3 - P1, P3 - P2
    v1c, v2c, v3c = P1 - X, P2 - X, P3 - X
    d2121, d2131, d2132 = dot(v21, v21), dot(v21, v31), dot(v21, v32)
    d3131, d3232, d3231 = dot(v31, v31), dot(v32, v32), dot(v32, v31)
    s21 = np.sqrt(d2121)
    d211c, d212c, d322c = dot(v21, v1c), dot(v21, v2c), dot(v32, v2c)
    d1c1c, d1c31, d2c2c, d2c1c = dot(v1c, v1c), dot(v1c, v31), dot(v2c, v2c), dot(v2c, v1c)
    d3c31, d3c32, d3c3c = dot(v3c, v31), dot(v3c, v32), dot(v3c, v3c)
    S = [np.zeros_like(d2121) for _ in range(7)]
    for y, w in zip(_GY, _GW):
        y, w = T(y), T(w)
        q1 = np.sqrt(d1c1c + 2 * y * d1c31 + y * y * d3131)
        q2 = np.sqrt(d2c2c + 2 * y * d322c + y * y * d3232)
        hv = np.log((d212c + d2132 * y + s21 * q2) / (d211c + d2131 * y + s21 * q1)) / s21
        hyc = (d211c * d211c - d1c1c * d2121 - 2 * y * d1c31 * d2121 + 2 * y * d211c * d2131 +
               y * y * d2131 * d2131 - y * y * d2121 * d3131)
        hyv = ((d211c + y * d2131) / q1 - (y * d2132 + d212c) / q2) / hyc
        hxyv = (q1 + (y * d211c - d2c1c - 2 * y * d1c31 - y * d2131 - y * y * d3231) / q2) / (-hyc)
        hxa = (-d1c31 - y * d2131) / np.sqrt(d1c1c + 2 * y * d211c + y * y * d2121)
        hxb = (d3c31 - y * d3231) / np.sqrt(y * y * d3232 - 2 * y * d3c32 + d3c3c)
        hxc = (d1c1c * d3131 - d1c31 * d1c31 + 2 * y * (d211c * d3131 - d1c31 * d2131) +
               y * y * (d2121 * d3131 - d2131 * d2131))
        hxv = (hxa + hxb) / hxc
        for k, v in enumerate((w * hv, w * hyv, w * hxyv, w * y * hyv, w * y * hxyv, w * y * y * hyv, w * y * y * hxv)):
            S[k] = S[k] + v
    t0, s0, sx, sy, sxy, syy, sxx = (v / 2 for v in S)
    out = np.empty((len(rows), 3, 3), dtype=np.float64)
    for a in range(3):
        for b in range(3):
            tt = (v1c[:, a] * v1c[:, b] * s0 + (v1c[:, a] * v21[:, b] + v21[:, a] * v1c[:, b]) * sx +
                  (v31[:, a] * v1c[:, b] + v1c[:, a] * v31[:, b]) * sy +
                  (v21[:, a] * v31[:, b] + v31[:, a] * v21[:, b]) * sxy +
                  v21[:, a] * v21[:, b] * sxx + v31[:, a] * v31[:, b] * syy)
            out[:, a, b] = (2 * area * ((t0 if a == b else 0) + T(cg) * tt)).astype(np.float64)
    return out


def diag_mean(self9, n):
    return lib().orc_diag_mean(n, _ptr(self9))


def deflate(s: Setup, gr, xmu, gdef):
    """best.f:406-425 in place on a full GR (column-major)."""
    comp = np.ascontiguousarray(s.icomp, dtype=np.int32)
    lib().orc_deflate(s.n, s.ndef, _ptr(np.ascontiguousarray(gdef)), comp.ctypes.data_as(_ip), _ptr(xmu),
                      gr.ctypes.data_as(_dp), gr.shape[0])


def ulp_hist(a, b, nb=8):
    """(histogram of ulp distances, worst) between two float64 arrays of equal size."""
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    b = np.ascontiguousarray(b, dtype=np.float64).ravel()
    h = np.zeros(nb, dtype=np.int64)
    w = lib().orc_ulp_hist(a.size, _ptr(a), _ptr(b), h.ctypes.data_as(_llp), nb)
    return h, int(w)


# ----------------------------------------------------------------------------------------------
# LAPACK (the reference's dgetrf/dgetrs)
# ----------------------------------------------------------------------------------------------

def getrf(gr):
    """dgetrf in place (best.f:444); returns (lu, ipiv 1-based, info)."""
    from scipy.linalg import lapack
    lu, piv, info = lapack.dgetrf(gr, overwrite_a=1)
    return lu, piv + 1, int(info)


def getrs(lu, ipiv, b):
    """dgetrs('N') (besolve.f90:133)."""
    from scipy.linalg import lapack
    x, info = lapack.dgetrs(lu, ipiv - 1, b)
    return x, int(info)


# ----------------------------------------------------------------------------------------------
# Post-processing (DIFCO, MATIN3, VISCO, JACOBI, OUTPUT)
# ----------------------------------------------------------------------------------------------

def rhs6(x, n):
    """difco.f:28-44: unit translations and rotations (omega x X) at the incenters."""
    X = x.reshape(3, n)
    B = np.zeros((3 * n, 6), order="F")
    B[0::3, 0] = 1.0
    B[1::3, 1] = 1.0
    B[2::3, 2] = 1.0
    B[1::3, 3] = -X[2]
    B[2::3, 3] = X[1]
    B[0::3, 4] = X[2]
    B[2::3, 4] = -X[0]
    B[0::3, 5] = -X[1]
    B[1::3, 5] = X[0]
    return B


def strain5(x, n):
    """visco.f:216-243: the five pure strain flows at the incenters."""
    X = x.reshape(3, n)
    V = np.zeros((3 * n, 5), order="F")
    V[0::3, 0] = 0.5 * X[1]
    V[1::3, 0] = 0.5 * X[0]
    V[0::3, 1] = 0.5 * X[2]
    V[2::3, 1] = 0.5 * X[0]
    V[1::3, 2] = 0.5 * X[2]
    V[2::3, 2] = 0.5 * X[1]
    V[0::3, 3] = 0.5 * X[0]
    V[1::3, 3] = -0.5 * X[1]
    V[0::3, 4] = 0.5 * X[0]
    V[2::3, 4] = -0.5 * X[2]
    return V


def matin3(A):
    """matin3.f: 3x3 inverse by Crout LU with implicit scaling (LUDCMP3) and back substitution
    (LUBKSB3).  A is indexed A[i][j] for Fortran A(i+1,j+1).  Returns (Y, ierr)."""
    cv = complex if np.iscomplexobj(np.asarray(A)) else float
    a = [[cv(A[i][j]) for j in range(3)] for i in range(3)]
    Y = [[1.0 if i == j else 0.0 for j in range(3)] for i in range(3)]
    n = 3
    TINY = 1e-20
    vv = [0.0] * 3
    ierr = 0
    for i in range(n):
        aamax = 0.0
        for j in range(n):
            if abs(_re(a[i][j])) > aamax:
                aamax = abs(_re(a[i][j]))
        if aamax == 0.0:
            ierr = 1
            aamax = 1.0
        vv[i] = 1.0 / aamax
    if ierr == 1:
        return np.array(Y), ierr
    indx = [0] * 3
    imax = 0
    for j in range(n):
        if j > 0:
            for i in range(j):
                s = a[i][j]
                if i > 0:
                    for k in range(i):
                        s = s - a[i][k] * a[k][j]
                    a[i][j] = s
        aamax = 0.0
        for i in range(j, n):
            s = a[i][j]
            if j > 0:
                for k in range(j):
                    s = s - a[i][k] * a[k][j]
                a[i][j] = s
            dum = vv[i] * abs(_re(s))
            if dum >= aamax:
                imax = i
                aamax = dum
        if j != imax:
            a[imax], a[j] = a[j], a[imax]
            vv[imax] = vv[j]
        indx[j] = imax
        if j != n - 1:
            if _re(a[j][j]) == 0.0:
                a[j][j] = TINY
            dum = 1.0 / a[j][j]
            for i in range(j + 1, n):
                a[i][j] = a[i][j] * dum
    if _re(a[n - 1][n - 1]) == 0.0:
        a[n - 1][n - 1] = TINY
    for col in range(n):
        b = [Y[r][col] for r in range(n)]
        ii = -1
        for i in range(n):
            ll = indx[i]
            s = b[ll]
            b[ll] = b[i]
            if ii != -1:
                for j in range(ii, i):
                    s = s - a[i][j] * b[j]
            elif _re(s) != 0.0:
                ii = i
            b[i] = s
        for i in range(n - 1, -1, -1):
            s = b[i]
            for j in range(i + 1, n):
                s = s - a[i][j] * b[j]
            b[i] = s / a[i][i]
        for r in range(n):
            Y[r][col] = b[r]
    return np.array(Y), ierr


def _m3(A, B):
    return [[sum_ordered([A[i][k] * B[k][j] for k in range(3)]) for j in range(3)] for i in range(3)]


def sum_ordered(terms):
    s = terms[0]
    for t in terms[1:]:
        s = s + t
    return s


def difco(B, x, area, n, cg=1.0):
    """difco.f:53-401 on the six solutions B (3n x 6).  Returns a dict of the friction and
    diffusion tensors (internal units) and the centre vectors."""
    X = x.reshape(3, n)
    dt = np.result_type(B, x, area)
    Ktt = np.zeros((3, 3), dtype=dt); Ktr = np.zeros((3, 3), dtype=dt); Krt = np.zeros((3, 3), dtype=dt); Krr = np.zeros((3, 3), dtype=dt)
    for mx in range(6):
        F = [B[0::3, mx], B[1::3, mx], B[2::3, mx]]
        TQ = [X[1] * F[2] - X[2] * F[1], X[2] * F[0] - X[0] * F[2], X[0] * F[1] - X[1] * F[0]]
        fto = [-_seqsum(area * F[c]) for c in range(3)]
        tto = [-_seqsum(area * TQ[c]) for c in range(3)]
        if mx < 3:
            i = mx
            temp = 1.0 / 1.0
            for j in range(3):
                Ktt[j, i] = -fto[j] * temp
                Ktr[j, i] = -tto[j] * temp
        else:
            i = mx - 3
            temp = 1.0 / 1.0
            for j in range(3):
                Krt[j, i] = -fto[j] * temp
                Krr[j, i] = -tto[j] * temp
    raw = dict(Ktt=Ktt.copy(), Ktr=Ktr.copy(), Krt=Krt.copy(), Krr=Krr.copy())
    uu = np.zeros((3, 3), dtype=dt)
    uu[0, 0] = Ktt[1, 1] + Ktt[2, 2]
    uu[1, 1] = Ktt[0, 0] + Ktt[2, 2]
    uu[2, 2] = Ktt[1, 1] + Ktt[0, 0]
    uu[0, 1] = -Ktt[0, 1]
    uu[0, 2] = -Ktt[0, 2]
    uu[2, 1] = -Ktt[1, 2]
    uu[1, 0] = uu[0, 1]
    uu[1, 2] = uu[2, 1]
    uu[2, 0] = uu[0, 2]
    Krt[0, 2] = (Krt[0, 2] + Ktr[2, 0]) * 0.5
    Krt[2, 0] = (Krt[2, 0] + Ktr[0, 2]) * 0.5
    Krt[0, 1] = (Krt[0, 1] + Ktr[1, 0]) * 0.5
    Krt[1, 0] = (Krt[1, 0] + Ktr[0, 1]) * 0.5
    Krt[1, 2] = (Krt[1, 2] + Ktr[2, 1]) * 0.5
    Krt[2, 1] = (Krt[2, 1] + Ktr[1, 2]) * 0.5
    Krt[0, 0] = (Krt[0, 0] + Ktr[0, 0]) * 0.5
    Krt[1, 1] = (Krt[1, 1] + Ktr[1, 1]) * 0.5
    Krt[2, 2] = (Krt[2, 2] + Ktr[2, 2]) * 0.5
    sur1 = -Krt[2, 1] + Krt[1, 2]
    sur2 = -Krt[0, 2] + Krt[2, 0]
    sur3 = -Krt[1, 0] + Krt[0, 1]
    aux, ierr = matin3(uu)
    urc = np.array([aux[j, 0] * sur1 + aux[j, 1] * sur2 + aux[j, 2] * sur3 for j in range(3)])
    uu = _antisym(urc)
    Krr_new = np.zeros((3, 3), dtype=dt)
    for i in range(3):
        for j in range(3):
            temp = 0.0
            for k in range(3):
                temp = temp + uu[i, k] * (Ktt[k, 0] * uu[0, j] + Ktt[k, 1] * uu[1, j] + Ktt[k, 2] * uu[2, j])
            temp1 = Krt[0, i] * uu[0, j] + Krt[1, i] * uu[1, j] + Krt[2, i] * uu[2, j]
            temp2 = uu[i, 0] * Krt[0, j] + uu[i, 1] * Krt[1, j] + uu[i, 2] * Krt[2, j]
            Krr_new[i, j] = Krr[i, j] - temp + temp1 - temp2
    Krr = Krr_new
    Krt_new = np.zeros((3, 3), dtype=dt)
    for i in range(3):
        for j in range(3):
            Krt_new[i, j] = Krt[i, j] + Ktt[i, 0] * uu[0, j] + Ktt[i, 1] * uu[1, j] + Ktt[i, 2] * uu[2, j]
    Krt = Krt_new
    Kttinv, _ = matin3(Ktt)
    KrrCR = Krr.copy()
    M = np.zeros((3, 3), dtype=dt)
    for i in range(3):
        for j in range(3):
            temp = 0.0
            for k in range(3):
                temp = temp + Krt[i, k] * (Kttinv[k, 0] * Krt[j, 0] + Kttinv[k, 1] * Krt[j, 1] + Kttinv[k, 2] * Krt[j, 2])
            M[i, j] = Krr[i, j] - temp
    Drr, _ = matin3(M)
    if cg == 0:
        Drr = 4.0 * Drr / 3.0
    Dtr = np.zeros((3, 3), dtype=dt)
    for i in range(3):
        for j in range(3):
            temp = 0.0
            for k in range(3):
                temp = temp + Kttinv[i, k] * (Krt[0, k] * Drr[0, j] + Krt[1, k] * Drr[1, j] + Krt[2, k] * Drr[2, j])
            Dtr[i, j] = -temp
            if cg == 0:
                Dtr[i, j] = 4.0 * Dtr[i, j] / 3.0
    Dtt = np.zeros((3, 3), dtype=dt)
    for i in range(3):
        for j in range(3):
            temp = 0.0
            for k in range(3):
                temp = temp + Kttinv[i, k] * (Krt[0, k] * Dtr[j, 0] + Krt[1, k] * Dtr[j, 1] + Krt[2, k] * Dtr[j, 2])
            Dtt[i, j] = Kttinv[i, j] - temp
            if cg == 0:
                Dtt[i, j] = 4.0 * Dtt[i, j] / 3.0
    uu = np.zeros((3, 3), dtype=dt)
    uu[0, 0] = Drr[1, 1] + Drr[2, 2]
    uu[1, 1] = Drr[0, 0] + Drr[2, 2]
    uu[2, 2] = Drr[1, 1] + Drr[0, 0]
    uu[0, 1] = -Drr[0, 1]
    uu[0, 2] = -Drr[0, 2]
    uu[2, 1] = -Drr[2, 1]
    uu[1, 0] = uu[0, 1]
    uu[1, 2] = uu[2, 1]
    uu[2, 0] = uu[0, 2]
    sur1 = Dtr[2, 1] - Dtr[1, 2]
    sur2 = Dtr[0, 2] - Dtr[2, 0]
    sur3 = Dtr[1, 0] - Dtr[0, 1]
    aux, _ = matin3(uu)
    udr = np.array([aux[j, 0] * sur1 + aux[j, 1] * sur2 + aux[j, 2] * sur3 for j in range(3)])
    uu = _antisym(udr)
    Dtt_new = np.zeros((3, 3), dtype=dt)
    for i in range(3):
        for j in range(3):
            temp = 0.0
            for k in range(3):
                temp = temp + uu[i, k] * Drr[k, 0] * uu[0, j] + uu[i, k] * Drr[k, 1] * uu[1, j] + uu[i, k] * Drr[k, 2] * uu[2, j]
            temp1 = Dtr[i, 0] * uu[0, j] + Dtr[i, 1] * uu[1, j] + Dtr[i, 2] * uu[2, j]
            temp2 = -uu[i, 0] * Dtr[j, 0] - uu[i, 1] * Dtr[j, 1] - uu[i, 2] * Dtr[j, 2]
            Dtt_new[i, j] = Dtt[i, j] - temp + temp1 + temp2
    Dtt = Dtt_new
    Dtr_new = np.zeros((3, 3), dtype=dt)
    for i in range(3):
        for j in range(3):
            Dtr_new[i, j] = Dtr[i, j] - uu[i, 0] * Drr[0, j] - uu[i, 1] * Drr[1, j] - uu[i, 2] * Drr[2, j]
    Dtr = Dtr_new
    return dict(Dtt=Dtt, Dtr=Dtr, Drr=Drr, urc=urc, udr=udr, Ktt=raw["Ktt"], KrtCR=Krt, KrrCR=KrrCR, raw=raw)


def _antisym(u):
    uu = np.zeros((3, 3), dtype=np.result_type(*[np.asarray(v) for v in u]))
    uu[2, 0] = -u[1]
    uu[2, 1] = u[0]
    uu[0, 1] = -u[2]
    uu[1, 0] = -uu[0, 1]
    uu[1, 2] = -uu[2, 1]
    uu[0, 2] = -uu[2, 0]
    return uu


def visco(V0, B, x, area, n, icov, cg=1.0):
    """visco.f:24-213 given V0 = solutions of the 5 strain flows and B[:, :3] the unit
    translations.  Returns (chiprime, (d1, d2, d3))."""
    X = x.reshape(3, n).copy()
    V0 = np.array(V0, order="F", copy=True)
    d1 = d2 = d3 = 0.0
    if icov:
        G = np.zeros((n, 5, 3))
        H = np.zeros((n, 5, 3, 3))
        for k in range(3):
            for l in range(5):
                G[:, l, k] = 2.0 * V0[k::3, l]
            E1, E2, E3 = B[k::3, 0], B[k::3, 1], B[k::3, 2]
            H[:, 0, k, 0] = E2; H[:, 0, k, 1] = E1; H[:, 0, k, 2] = 0.0
            H[:, 1, k, 0] = E3; H[:, 1, k, 1] = 0.0; H[:, 1, k, 2] = E1
            H[:, 2, k, 0] = 0.0; H[:, 2, k, 1] = E3; H[:, 2, k, 2] = E2
            H[:, 3, k, 0] = E1; H[:, 3, k, 1] = -E2; H[:, 3, k, 2] = 0.0
            H[:, 4, k, 0] = E1; H[:, 4, k, 1] = 0.0; H[:, 4, k, 2] = -E3
        h = lambda l, k, m: H[:, l - 1, k - 1, m - 1]  # noqa: E731  (Fortran 1-based H(N,L,K,M))
        g = lambda l, k: G[:, l - 1, k - 1]  # noqa: E731
        A = area
        BB = np.zeros((3, 3))
        BB[0, 0] = _seqsum(A * (3 * (h(1, 2, 1) + h(2, 3, 1)) + 2 * (h(4, 1, 1) + h(5, 1, 1))))
        BB[0, 1] = _seqsum(A * (-4 * h(4, 2, 1) + 3 * (h(1, 1, 1) + h(1, 2, 2) + h(2, 3, 2) + h(3, 3, 1))
                                + 2 * (h(4, 1, 2) + h(5, 1, 2) + h(5, 2, 1))))
        BB[0, 2] = _seqsum(A * (-4 * h(5, 3, 1) + 3 * (h(1, 2, 3) + h(2, 1, 1) + h(2, 3, 3) + h(3, 2, 1))
                                + 2 * (h(4, 1, 3) + h(4, 3, 1) + h(5, 1, 3))))
        BB[1, 1] = _seqsum(A * (-4 * h(4, 2, 2) + 3 * (h(1, 1, 2) + h(3, 3, 2)) + 2 * h(5, 2, 2)))
        BB[1, 2] = _seqsum(A * (-4 * h(4, 2, 3) + 3 * (h(3, 2, 2) + h(3, 3, 3) + h(1, 1, 3) + h(2, 1, 2))
                                + 2 * (h(4, 3, 2) + h(5, 2, 3))))
        BB[2, 2] = _seqsum(A * (-4 * h(5, 3, 3) + 3 * (h(2, 1, 3) + h(3, 2, 3)) + 2 * h(4, 3, 3)))
        x1, x2, x3 = X[0], X[1], X[2]
        C1 = _seqsum(A * (-3 * g(1, 2) - 3 * g(2, 3) - 2 * g(4, 1) - 2 * g(5, 1)
                          - x1 * (3 * (h(1, 2, 1) + h(2, 3, 1)) + 2 * (h(4, 1, 1) + h(5, 1, 1)))
                          - x2 * (3 * (h(1, 1, 1) + h(3, 3, 1)) - 4 * h(4, 2, 1) + 2 * h(5, 2, 1))
                          - x3 * (3 * (h(2, 1, 1) + h(3, 2, 1)) - 4 * h(5, 3, 1) + 2 * h(4, 3, 1))))
        C2 = _seqsum(A * (-3 * g(1, 1) - 3 * g(3, 3) + 4 * g(4, 2) - 2 * g(5, 2)
                          - x1 * (3 * (h(1, 2, 2) + h(2, 3, 2)) + 2 * (h(4, 1, 2) + h(5, 1, 2)))
                          - x2 * (3 * (h(1, 1, 2) + h(3, 3, 2)) - 4 * h(4, 2, 2) + 2 * h(5, 2, 2))
                          - x3 * (3 * (h(2, 1, 2) + h(3, 2, 2)) - 4 * h(5, 3, 2) + 2 * h(4, 3, 2))))
        C3 = _seqsum(A * (-3 * g(2, 1) - 3 * g(3, 2) - 2 * g(4, 3) + 4 * g(5, 3)
                          - x1 * (3 * (h(1, 2, 3) + h(2, 3, 3)) + 2 * (h(4, 1, 3) + h(5, 1, 3)))
                          - x2 * (3 * (h(1, 1, 3) + h(3, 3, 3)) - 4 * h(4, 2, 3) + 2 * h(5, 2, 3))
                          - x3 * (3 * (h(2, 1, 3) + h(3, 2, 3)) - 4 * h(5, 3, 3) + 2 * h(4, 3, 3))))
        BB[0, 0] = BB[0, 0] / 15.
        BB[0, 1] = BB[0, 1] / 30.
        BB[0, 2] = BB[0, 2] / 30.
        BB[1, 0] = BB[0, 1]
        BB[1, 1] = BB[1, 1] / 15.
        BB[1, 2] = BB[1, 2] / 30.
        BB[2, 0] = BB[0, 2]
        BB[2, 1] = BB[1, 2]
        BB[2, 2] = BB[2, 2] / 15.
        C1, C2, C3 = C1 / 30., C2 / 30., C3 / 30.
        BBI, _ = matin3(BB)
        d1 = BBI[0, 0] * C1 + BBI[0, 1] * C2 + BBI[0, 2] * C3
        d2 = BBI[1, 0] * C1 + BBI[1, 1] * C2 + BBI[1, 2] * C3
        d3 = BBI[2, 0] * C1 + BBI[2, 1] * C2 + BBI[2, 2] * C3
        X[0] = X[0] - d1
        X[1] = X[1] - d2
        X[2] = X[2] - d3
        E1, E2, E3 = B[:, 0], B[:, 1], B[:, 2]
        V0[:, 0] = V0[:, 0] - 0.5 * (d2 * E1 + d1 * E2)
        V0[:, 1] = V0[:, 1] - 0.5 * (d3 * E1 + d1 * E3)
        V0[:, 2] = V0[:, 2] - 0.5 * (d3 * E2 + d2 * E3)
        V0[:, 3] = V0[:, 3] - 0.5 * (d1 * E1 - d2 * E2)
        V0[:, 4] = V0[:, 4] - 0.5 * (d1 * E1 - d3 * E3)
    W = lambda l, c: V0[c - 1::3, l - 1]  # noqa: E731  W(L, I0+c)
    A = area
    chi112 = 0.5 * _seqsum(A * (W(1, 1) * X[1] + W(1, 2) * X[0]))
    chi213 = 0.5 * _seqsum(A * (W(2, 1) * X[2] + W(2, 3) * X[0]))
    chi323 = 0.5 * _seqsum(A * (W(3, 2) * X[2] + W(3, 3) * X[1]))
    chi411 = _seqsum(A * W(4, 1) * X[0])
    chi422 = _seqsum(A * W(4, 2) * X[1])
    chi433 = _seqsum(A * W(4, 3) * X[2])
    chi511 = _seqsum(A * W(5, 1) * X[0])
    chi522 = _seqsum(A * W(5, 2) * X[1])
    chi533 = _seqsum(A * W(5, 3) * X[2])
    PI = 3.1415926535897932385
    chip = 8 * PI * (0.2 * (chi112 + chi213 + chi323)
                     + (chi411 - 2 * chi422 + chi433 + chi511 + chi522 - 2 * chi533) / 15.0)
    if cg == 0:
        chip = 0.75 * chip
    return chip, (d1, d2, d3)


def jacobi3(a):
    """jacobi.f: cyclic Jacobi eigenvalues of a symmetric 3x3 (uses the upper triangle)."""
    a = [[float(a[i][j]) for j in range(3)] for i in range(3)]
    n = 3
    v = [[1.0 if i == j else 0.0 for j in range(3)] for i in range(3)]
    b = [a[i][i] for i in range(3)]
    d = list(b)
    z = [0.0] * 3
    for it in range(1, 51):
        sm = 0.0
        for ip in range(n - 1):
            for iq in range(ip + 1, n):
                sm = sm + abs(a[ip][iq])
        if sm == 0.0:
            return np.array(d)
        tresh = 0.2 * sm / n ** 2 if it < 4 else 0.0
        for ip in range(n - 1):
            for iq in range(ip + 1, n):
                g = 100. * abs(a[ip][iq])
                if it > 4 and abs(d[ip]) + g == abs(d[ip]) and abs(d[iq]) + g == abs(d[iq]):
                    a[ip][iq] = 0.0
                elif abs(a[ip][iq]) > tresh:
                    h = d[iq] - d[ip]
                    if abs(h) + g == abs(h):
                        t = a[ip][iq] / h
                    else:
                        theta = 0.5 * h / a[ip][iq]
                        t = 1. / (abs(theta) + np.sqrt(1. + theta * theta))
                        if theta < 0.0:
                            t = -t
                    c = 1. / np.sqrt(1 + t * t)
                    s = t * c
                    tau = s / (1. + c)
                    h = t * a[ip][iq]
                    z[ip] -= h
                    z[iq] += h
                    d[ip] -= h
                    d[iq] += h
                    a[ip][iq] = 0.0
                    for j in range(0, ip):
                        g, h = a[j][ip], a[j][iq]
                        a[j][ip] = g - s * (h + g * tau)
                        a[j][iq] = h + s * (g - h * tau)
                    for j in range(ip + 1, iq):
                        g, h = a[ip][j], a[j][iq]
                        a[ip][j] = g - s * (h + g * tau)
                        a[j][iq] = h + s * (g - h * tau)
                    for j in range(iq + 1, n):
                        g, h = a[ip][j], a[iq][j]
                        a[ip][j] = g - s * (h + g * tau)
                        a[iq][j] = h + s * (g - h * tau)
                    for j in range(n):
                        g, h = v[j][ip], v[j][iq]
                        v[j][ip] = g - s * (h + g * tau)
                        v[j][iq] = h + s * (g - h * tau)
        for ip in range(n):
            b[ip] = b[ip] + z[ip]
            d[ip] = b[ip]
            z[ip] = 0.0
    return np.array(d)


# output.f:16-29 (the constants exactly as written there)
TEMPERATURE = 293.15
ETA_POISE = 0.01002
PI_OUT = 3.141592653
TUNIT = (1.38066E-16) * TEMPERATURE * 1.0E8 / (8.0 * ETA_POISE * PI_OUT)
RUNIT = TUNIT * 1.0e16


def report(d, chiprime=None, truevol=None, wm=None, iarea=1):
    """output.f:96-171: eigenvalue traces in cgs units, CHI and [eta]."""
    ev_r = jacobi3(d["Drr"])
    ev_t = jacobi3(d["Dtt"])
    out = dict(trace_drr=(ev_r[0] + ev_r[1] + ev_r[2]) / 3.0, trace_dtt=(ev_t[0] + ev_t[1] + ev_t[2]) / 3.0)
    out["DR"] = RUNIT * out["trace_drr"]
    out["DTRANS"] = TUNIT * out["trace_dtt"]
    if chiprime is not None:
        out["chiprime"] = chiprime
        if iarea and truevol:
            out["CHI"] = chiprime / truevol
        if wm:
            out["ETA"] = chiprime * 0.602214 / wm
    return out


@dataclass
class Result:
    setup: Setup
    x: np.ndarray
    diagm: float
    xmu: np.ndarray
    gdef: np.ndarray
    B6: np.ndarray
    tensors: dict
    report: dict
    V5: np.ndarray = None
    chiprime: float = None
    dvisc: tuple = None
    info: int = 0


def best_run(tri, truearea=None, truevol=None, iarea=1, cg=1.0, ivisco=0, icov=0, wm=None, use_ref=False):
    """The whole dense path on the CPU (best.f:184-498 without the file output)."""
    s = setup(tri, iarea, truearea)
    if use_ref:
        gr, x, dm = assemble_ref(s, cg)
    else:
        gr, x, self9 = assemble(s, cg)
        dm = diag_mean(self9, s.n)
    xmu, gdef = deflation_vectors(s, dm)
    deflate(s, gr, xmu, gdef)
    lu, ipiv, info = getrf(gr)
    del gr
    B = rhs6(x, s.n)
    B6, _ = getrs(lu, ipiv, B)
    t = difco(B6, x, s.area, s.n, cg)
    res = Result(setup=s, x=x, diagm=dm, xmu=xmu, gdef=gdef, B6=B6, tensors=t, report=None, info=info)
    chip = None
    if ivisco:
        V5, _ = getrs(lu, ipiv, strain5(x, s.n))
        chip, dv = visco(V5, B6, x, s.area, s.n, icov, cg)
        res.V5, res.chiprime, res.dvisc = V5, chip, dv
    res.report = report(t, chip, truevol, wm, iarea)
    return res
