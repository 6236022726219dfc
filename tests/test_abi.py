"""CPU tests of the boundary: libbestgpu builds for sm_100a, loads, and exports every function that
include/*.h declares; without a GPU it reports itself unavailable and refuses work (there is no CPU
path behind the seam)."""
import ctypes
import os
import re

import pytest

import best_hydro_b200 as bh
from best_hydro_b200 import build as bbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b((?:bhm|bgpu)_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_builds_and_exports_every_declared_symbol():
    path = bbuild.build()
    assert os.path.exists(path)
    L = ctypes.CDLL(path)
    names = declared_functions()
    assert len(names) >= 9
    for nm in names:
        assert hasattr(L, nm), nm
    # the nine functions BEST binds (best/besolve.f90:48-89)
    for nm in ("bhm_available", "bhm_create", "bhm_incenters", "bhm_entries", "bhm_diag_mean", "bhm_build",
               "bhm_solve", "bhm_log_line", "bhm_destroy"):
        assert nm in names


def test_python_mirror_covers_the_header():
    assert set(declared_functions()) == set(bh._SIGS)


def test_oracle_libraries_export():
    from oracle import best as ob
    L = ob.lib()
    for nm in ("orc_self_blocks", "orc_gr_block", "orc_diag_mean", "orc_deflate", "orc_ulp_hist"):
        assert hasattr(L, nm)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour without a GPU")
def test_no_gpu_means_unavailable_and_no_cpu_fallback():
    import numpy as np
    assert bh.BhmSolver.available() is False
    s = bh.BhmSolver()
    v = np.zeros(9)
    with pytest.raises(bh.BestGpuError, match="CUDA"):
        s.create(v, v, v, np.ones(3), 1.0)


def test_log_queue_is_empty_or_drains():
    bh.log_lines()
    assert bh.lib().bhm_log_line(ctypes.create_string_buffer(8), 8) == -1
