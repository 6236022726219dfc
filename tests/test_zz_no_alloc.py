"""bgpu_dgetrs_noalloc: the solve for callers that cannot allocate GPU memory (an application whose
pool allocator owns all device memory, or that forbids a library to allocate behind its back).  It
must give what the allocating solve bgpu_dgetrs_device gives, on two calls in a row (the second
reuses the fixed scratch the first left behind), and refuse orders its fixed scratch cannot hold.
Collected last so that a failure here stops a -x run only after every other test has run."""
import ctypes

import numpy as np
import pytest

import best_hydro_b200 as bh

pytestmark = pytest.mark.gpu
TOL = 1e-11  # the solve tolerance of tests/test_gpu_lu.py


def _dev(torch, a):
    m, n = a.shape
    ld = m + (m & 1)
    t = torch.zeros((n, ld), dtype=torch.float64)
    t[:, :m] = torch.from_numpy(np.ascontiguousarray(a.T))
    t = t.cuda()
    torch.cuda.synchronize()
    return t, ld


def test_noalloc_solve_matches_allocating_solve_twice():
    import torch
    assert torch.cuda.is_available()
    rng = np.random.default_rng(7)
    n = 2500
    A = np.asfortranarray(rng.standard_normal((n, n)) + np.sqrt(n) * np.eye(n))
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
        x1 = d1[:, :n].cpu().numpy()
        x2 = d2[:, :n].cpu().numpy()
        err = np.max(np.abs(x2 - x1)) / np.max(np.abs(x1))
        assert err < TOL, (call, err)


def test_noalloc_rejects_orders_beyond_its_scratch():
    bh.log_lines()
    n = 1_000_000
    rc = bh.lib().bgpu_dgetrs_noalloc(n, 6, None, n, None, None, n, None)
    assert rc != 0
    msgs = " ".join(bh.log_lines())
    assert "exceeds" in msgs and "MiB" in msgs
