"""bgpu_dgetrs_noalloc: the solve for callers that cannot allocate GPU memory -- an application whose
own pool allocator has reserved the device's memory, or that forbids a library to allocate behind
its back.  Its scratch is a fixed array in the library's device image.

Checked here: on two calls in a row (6, then 11 right-hand sides; the second reuses the scratch the
first left behind) its solutions equal the allocating solve bgpu_dgetrs_device's and LAPACK's
(scipy) within the solve tolerance of tests/test_gpu_lu.py, with small residuals; with CUDA's lazy
module loading, a warm-up call (n = 0) made first lets a later solve run after the application has
taken nearly all free memory, without the free memory changing; orders its array cannot hold are
refused.  Collected last so that a failure here stops a -x run only after every other test has run.
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import scipy.linalg

import best_hydro_b200 as bh

pytestmark = pytest.mark.gpu
TOL = 1e-11  # the solve tolerance of tests/test_gpu_lu.py
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _dev(torch, a):
    m, n = a.shape
    ld = m + (m & 1)
    t = torch.zeros((n, ld), dtype=torch.float64)
    t[:, :m] = torch.from_numpy(np.ascontiguousarray(a.T))
    t = t.cuda()
    torch.cuda.synchronize()
    return t, ld


def test_noalloc_solve_matches_lapack_and_allocating_solve_twice():
    import torch
    assert torch.cuda.is_available()
    rng = np.random.default_rng(7)
    n = 2500
    A = np.asfortranarray(rng.standard_normal((n, n)) + np.sqrt(n) * np.eye(n))
    lu_piv = scipy.linalg.lu_factor(A)
    dA, lda = _dev(torch, A)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert bh.dgetrf_device(n, dA.data_ptr(), lda, ipiv.data_ptr()) == 0
    for call, nrhs in enumerate((6, 11)):
        B = np.asfortranarray(rng.standard_normal((n, nrhs)))
        d1, ld = _dev(torch, B)
        d2, _ = _dev(torch, B)
        bh.dgetrs_device(n, nrhs, dA.data_ptr(), lda, ipiv.data_ptr(), d1.data_ptr(), ld)
        bh.dgetrs_noalloc(n, nrhs, dA.data_ptr(), lda, ipiv.data_ptr(), d2.data_ptr(), ld, 0)
        x1 = d1[:, :n].cpu().numpy().T
        x2 = d2[:, :n].cpu().numpy().T
        want = scipy.linalg.lu_solve(lu_piv, B)
        scale = np.max(np.abs(want))
        assert np.max(np.abs(x2 - want)) / scale < TOL, call
        assert np.max(np.abs(x2 - x1)) / scale < TOL, call
        res = np.max(np.abs(A @ x2 - B)) / (np.max(np.abs(A)) * np.max(np.abs(x2)) * n)
        assert res < 1e-15, (call, res)


_LAZY = r"""
import numpy as np, scipy.linalg, torch
import best_hydro_b200 as bh
n, nrhs = 700, 6
rng = np.random.default_rng(3)
A = rng.standard_normal((n, n)) + np.sqrt(n) * np.eye(n)
B = rng.standard_normal((n, nrhs))
dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
torch.cuda.synchronize()
assert bh.dgetrf_device(n, dA.data_ptr(), n, ipiv.data_ptr()) == 0
torch.cuda.synchronize()
# the warm-up, before the application's pool takes the memory
assert bh.lib().bgpu_dgetrs_noalloc(0, 6, None, 1, None, None, 1, None) == 0, bh.log_lines()
free, total = torch.cuda.mem_get_info()
pool = torch.empty(free - (48 << 20), dtype=torch.uint8, device="cuda")
torch.cuda.synchronize()
before, _ = torch.cuda.mem_get_info()
bh.dgetrs_noalloc(n, nrhs, dA.data_ptr(), n, ipiv.data_ptr(), dB.data_ptr(), n, 0)
after, _ = torch.cuda.mem_get_info()
x = dB.cpu().numpy().T
want = scipy.linalg.solve(A, B)
err = np.max(np.abs(x - want)) / np.max(np.abs(want))
assert err < 1e-11, err
assert before == after, (before, after)
print("lazy-loading warm-up ok", before >> 20, "MiB free, error", err)
"""


def test_noalloc_warm_up_under_lazy_module_loading():
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    r = subprocess.run([sys.executable, "-c", _LAZY], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "warm-up ok" in r.stdout


def test_noalloc_rejects_orders_beyond_its_scratch():
    bh.log_lines()
    n = 1_000_000
    rc = bh.lib().bgpu_dgetrs_noalloc(n, 6, None, n, None, None, n, None)
    assert rc != 0
    msgs = " ".join(bh.log_lines())
    assert "exceeds" in msgs and "MiB" in msgs
