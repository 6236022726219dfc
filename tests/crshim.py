"""Builds and loads tests/native/tgetgr_cr_shim.cpp: the oracle's TGETGR restatement with correctly
rounded transcendental functions, and its probe build that counts glibc's not-correctly-rounded
results per triangle pair (see that file)."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_L = None
_P = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_long)


def _build(name, extra):
    d = tempfile.mkdtemp()
    so = os.path.join(d, name)
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c++17", "-fpermissive", "-w"] + extra +
                   ["-o", so, os.path.join(HERE, "native", "tgetgr_cr_shim.cpp")], check=True)
    return ctypes.CDLL(so)


def lib():
    global _L
    if _L is None:
        L = _build("tgetgr_cr.so", ["-fopenmp"])
        L.orc_cr_self_blocks.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
        L.orc_cr_gr_block.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, _dp, _dp,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_long]
        _L = L
    return _L


def probe_lib():
    global _P
    if _P is None:
        P = _build("tgetgr_probe.so", ["-DBGPU_FN_PROBE"])
        P.orc_pr_fn_misrounds.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp,
                                          ctypes.c_long, _ip, _ip, _lp]
        _P = P
    return _P


def self_blocks_cr(s, cg=1.0):
    """(incenters, self9) with correctly rounded transcendentals, for an oracle Setup."""
    v1, v2, v3 = s.colmajor()
    x = np.empty(3 * s.n)
    self9 = np.empty(9 * s.n)
    lib().orc_cr_self_blocks(s.n, v1.ctypes.data_as(_dp), v2.ctypes.data_as(_dp), v3.ctypes.data_as(_dp), s.afac, cg,
                             x.ctypes.data_as(_dp), self9.ctypes.data_as(_dp))
    return x, self9


def assemble_cr(s, cg=1.0):
    """GR before deflation (column-major) with correctly rounded functions throughout: TGETGR's
    arithmetic as the GPU's exact kernels evaluate it.  Returns (gr, x, self9)."""
    v1, v2, v3 = s.colmajor()
    x, self9 = self_blocks_cr(s, cg)
    m = 3 * s.n
    gr = np.empty((m, m), dtype=np.float64, order="F")
    lib().orc_cr_gr_block(s.n, v1.ctypes.data_as(_dp), v2.ctypes.data_as(_dp), v3.ctypes.data_as(_dp),
                          s.area.ctypes.data_as(_dp), cg, x.ctypes.data_as(_dp), self9.ctypes.data_as(_dp),
                          0, s.n, 0, s.n, gr.ctypes.data_as(_dp), m)
    return gr, x, self9


def fn_misrounds(s, x, n1, n2, cg=1.0):
    """Per triangle pair (n1[k], n2[k]): how many of the acos/sin/cos/log calls of its GR block return,
    in glibc, a result that is not the correctly rounded one.  x: the reference's incenters."""
    v1, v2, v3 = s.colmajor()
    n1 = np.ascontiguousarray(n1, dtype=np.int32)
    n2 = np.ascontiguousarray(n2, dtype=np.int32)
    out = np.zeros(n1.size, dtype=np.int64)
    probe_lib().orc_pr_fn_misrounds(s.n, v1.ctypes.data_as(_dp), v2.ctypes.data_as(_dp), v3.ctypes.data_as(_dp),
                                    s.area.ctypes.data_as(_dp), s.afac, cg, np.ascontiguousarray(x).ctypes.data_as(_dp),
                                    n1.size, n1.ctypes.data_as(_ip), n2.ctypes.data_as(_ip), out.ctypes.data_as(_lp))
    return out


def block_scale_ulps(a9, b9):
    """Per entry, |a - b| in ulps of the largest entry of its 3x3 self block."""
    a9 = np.asarray(a9).reshape(-1, 9)
    b9 = np.asarray(b9).reshape(-1, 9)
    scale = np.max(np.abs(b9), axis=1, keepdims=True)
    return np.abs(a9 - b9) / np.spacing(scale)
