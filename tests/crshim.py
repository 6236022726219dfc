"""Builds and loads tests/native/tgetgr_cr_shim.cpp: the oracle's TGETGR restatement with correctly
rounded transcendental functions (see that file)."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_L = None


def lib():
    global _L
    if _L is None:
        d = tempfile.mkdtemp()
        so = os.path.join(d, "tgetgr_cr.so")
        subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c++17", "-fpermissive", "-w",
                        "-o", so, os.path.join(HERE, "native", "tgetgr_cr_shim.cpp")], check=True)
        L = ctypes.CDLL(so)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_cr_self_blocks.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_double, ctypes.c_double, dp, dp]
        _L = L
    return _L


def self_blocks_cr(s, cg=1.0):
    """(incenters, self9) with correctly rounded transcendentals, for an oracle Setup."""
    dp = ctypes.POINTER(ctypes.c_double)
    v1, v2, v3 = s.colmajor()
    x = np.empty(3 * s.n)
    self9 = np.empty(9 * s.n)
    lib().orc_cr_self_blocks(s.n, v1.ctypes.data_as(dp), v2.ctypes.data_as(dp), v3.ctypes.data_as(dp), s.afac, cg,
                             x.ctypes.data_as(dp), self9.ctypes.data_as(dp))
    return x, self9


def block_scale_ulps(a9, b9):
    """Per entry, |a - b| in ulps of the largest entry of its 3x3 self block."""
    a9 = np.asarray(a9).reshape(-1, 9)
    b9 = np.asarray(b9).reshape(-1, 9)
    scale = np.max(np.abs(b9), axis=1, keepdims=True)
    return np.abs(a9 - b9) / np.spacing(scale)
