"""ORACLE (test infrastructure only): the CPU reference gradient of BEST's D_t, D_r and CHI' with
respect to mesh vertex coordinates, by complex-step differentiation of the oracle's own pipeline.

For an analytic f, df/dx = Im f(x + i h) / h up to rounding for any tiny h (the complex-step
method: Squire and Trapp, SIAM Review 40 (1998) 110; Martins, Sturdza and Alonso, ACM TOMS 29 (2003)
245).  Every stage of the oracle is run in double complex: the set-up (best/best.f:261-315), the
assembly (oracle/tgetgr.c built with -DORC_COMPLEX -> lib/liborc_cs.so), the deflation
(best/best.f:384-426), the LU and solves (LAPACK zgetrf/zgetrs through scipy: the partial pivoting
follows the real parts, whose magnitudes the i h perturbation does not change), DIFCO and VISCO
(oracle/best.py, whose 3x3 inversions pivot on real parts).  Triangle connectivity (COMPON) is taken
from the real coordinates.  Only tests/ use this module; it is independent of the CUDA adjoint.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import scipy.linalg

from oracle import best as ob

HERE = os.path.dirname(os.path.abspath(__file__))
_CS = None
_dp = ctypes.POINTER(ctypes.c_double)

TUNIT = 1.38066e-16 * 293.15 * 1.0e8 / (8.0 * 0.01002 * 3.141592653)  # best/output.f:16-29
RUNIT = TUNIT * 1.0e16


def lib_cs():
    global _CS
    if _CS is None:
        path = os.path.join(HERE, "lib", "liborc_cs.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        L = ctypes.CDLL(path)
        L.orc_cs_self_blocks.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, _dp, _dp]
        L.orc_cs_gr_block.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_long]
        _CS = L
    return _CS


def _p(a):
    assert a.dtype == np.complex128 and a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def values(tri, iarea, truearea, cg=1.0):
    """D_t (cm^2/s), D_r (1/s) and CHI' (A^3, icov = 0) of a triangle soup tri (N x 9, complex)."""
    tri = np.asarray(tri, dtype=np.complex128)
    n = tri.shape[0]
    v1, v2, v3 = tri[:, 0:3].copy(), tri[:, 3:6].copy(), tri[:, 6:9].copy()
    for c in range(3):
        cen = ob._seqsum((v1[:, c] + v2[:, c] + v3[:, c]) / 3.0) / n
        v1[:, c] -= cen
        v2[:, c] -= cen
        v3[:, c] -= cen
    e21, e31 = v2 - v1, v3 - v1
    cr = np.stack([e31[:, 1] * e21[:, 2] - e31[:, 2] * e21[:, 1], e31[:, 2] * e21[:, 0] - e31[:, 0] * e21[:, 2],
                   e31[:, 0] * e21[:, 1] - e31[:, 1] * e21[:, 0]], axis=1)
    xnl = np.sqrt((cr * cr).sum(axis=1))
    area = xnl * 0.5
    afac = truearea / ob._seqsum(area) if iarea else 1.0
    area = afac * area
    # connectivity from the real coordinates (best/compon.f90)
    s_real = ob.setup(tri.real, 0, None)
    ndef, icomp = s_real.ndef, s_real.icomp
    L = lib_cs()
    cm = [np.ascontiguousarray(v.T).ravel() for v in (v1, v2, v3)]
    x = np.empty(3 * n, dtype=np.complex128)
    self9 = np.empty(9 * n, dtype=np.complex128)
    af = np.array([complex(afac).real, complex(afac).imag])
    L.orc_cs_self_blocks(n, _p(cm[0]), _p(cm[1]), _p(cm[2]), af.ctypes.data_as(_dp), cg, _p(x), _p(self9))
    gr = np.empty((3 * n, 3 * n), dtype=np.complex128, order="F")
    L.orc_cs_gr_block(n, _p(cm[0]), _p(cm[1]), _p(cm[2]), _p(np.ascontiguousarray(area)), cg, _p(x), _p(self9), 0, n,
                      0, n, gr.ctypes.data_as(_dp), 3 * n)
    diagm = ob._seqsum(self9.reshape(n, 9)[:, [0, 4, 8]].ravel()) / (3 * n)
    # deflation: XMU = area * unit normal, GDEF = DIAGM / |XMU|^2 per surface
    xmu = (area[:, None] * cr / xnl[:, None]).ravel()
    surf = icomp - 1 if ndef > 1 else np.zeros(n, dtype=int)
    for d in range(max(ndef, 1)):
        idx = np.nonzero(surf == d)[0]
        rows = (3 * idx[:, None] + np.arange(3)).ravel()
        xd = xmu[rows]
        gdef = diagm / (xd * xd).sum()
        gr[np.ix_(rows, rows)] += gdef * np.outer(xd, xd)
    B6 = np.zeros((3 * n, 6), dtype=np.complex128)
    X = x.reshape(3, n)
    B6[0::3, 0] = B6[1::3, 1] = B6[2::3, 2] = 1.0
    B6[1::3, 3], B6[2::3, 3] = -X[2], X[1]
    B6[0::3, 4], B6[2::3, 4] = X[2], -X[0]
    B6[0::3, 5], B6[1::3, 5] = -X[1], X[0]
    V5 = np.zeros((3 * n, 5), dtype=np.complex128)
    V5[0::3, 0], V5[1::3, 0] = 0.5 * X[1], 0.5 * X[0]
    V5[0::3, 1], V5[2::3, 1] = 0.5 * X[2], 0.5 * X[0]
    V5[1::3, 2], V5[2::3, 2] = 0.5 * X[2], 0.5 * X[1]
    V5[0::3, 3], V5[1::3, 3] = 0.5 * X[0], -0.5 * X[1]
    V5[0::3, 4], V5[2::3, 4] = 0.5 * X[0], -0.5 * X[2]
    lu = scipy.linalg.lu_factor(gr, check_finite=False)
    sol = scipy.linalg.lu_solve(lu, np.hstack([B6, V5]), check_finite=False)
    t = ob.difco(sol[:, :6], x, area, n, cg)
    chip, _ = ob.visco(sol[:, 6:], sol[:, :6], x, area, n, 0, cg)
    return np.array([TUNIT * np.trace(t["Dtt"]) / 3.0, RUNIT * np.trace(t["Drr"]) / 3.0, chip])


def gradient(verts, faces, iarea, truearea, picks, cg=1.0):
    """d(D_t, D_r, CHI') / d verts[v, c] for each (v, c) in picks, by complex step: array (3, len(picks))."""
    verts = np.asarray(verts, dtype=np.float64)
    scale = float(np.abs(verts).max())
    h = 1e-20 * scale
    out = np.empty((3, len(picks)))
    for k, (v, c) in enumerate(picks):
        vc = verts.astype(np.complex128)
        vc[v, c] += 1j * h
        tri = np.concatenate([vc[faces[:, 0]], vc[faces[:, 1]], vc[faces[:, 2]]], axis=1)
        out[:, k] = values(tri, iarea, truearea, cg).imag / h
    return out
