"""The failure path of a bounded device-side wait, exercised without a fault or a hang: with the
triangular solves' poll limit set to 0 (bgpu_set_wait_limit), a solve whose block rows wait for the
rows before them gives up at its first unsatisfied wait, the kernel records the timeout and returns,
and bhm_solve fails with the message; with the limit restored the same solver solves again, bit for
bit as before."""
import numpy as np
import pytest

import best_hydro_b200 as bh
from best_hydro_b200 import meshes

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_recoverable():
    tri, ta, tv = meshes.ellipsoid(16)  # 15,360 unknowns: 120 block rows, each waiting on the last
    st = bh.Setup(tri, 1, ta)
    s = bh.BhmSolver()
    s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = s.incenters()
    xmu, gdef = st.deflation(s.diag_mean())
    bh.set_precision(bh.BGPU_FP64)
    try:
        s.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        rhs = bh.rhs6(x)
        want = s.solve(rhs)
        bh.log_lines()
        assert bh.lib().bgpu_set_wait_limit(0) == 0
        try:
            with pytest.raises(bh.BestGpuError) as failure:
                s.solve(rhs)
        finally:
            assert bh.lib().bgpu_set_wait_limit(1 << 22) == 0
        assert "wait ran out" in str(failure.value), str(failure.value)
        again = s.solve(rhs)
        assert np.array_equal(again.view(np.int64), want.view(np.int64))
    finally:
        bh.set_precision(-1)
        s.destroy()
