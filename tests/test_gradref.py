"""The CPU reference gradient (oracle/gradref.py, complex step through the oracle's pipeline) checked
on the CPU: its values are the oracle's real results, and its derivatives agree with central
differences of the oracle's real pipeline."""
import numpy as np

from best_hydro_b200 import meshes
from oracle import best as ob
from oracle import gradref


def test_complex_pipeline_values_are_the_oracle_results():
    v, f, ta, tv = meshes.ellipsoid_vf(3)
    tri = meshes.to_triangles(v, f)
    val = gradref.values(tri.astype(complex), 1, ta)
    o = ob.best_run(tri, ta, tv, iarea=1, ivisco=1)
    assert np.all(np.abs(val.imag) == 0)
    ref = np.array([o.report["DTRANS"], o.report["DR"], o.chiprime])
    assert np.allclose(val.real, ref, rtol=1e-12, atol=0)


def test_complex_step_matches_central_differences():
    v, f, ta, tv = meshes.ellipsoid_vf(3)
    picks = [(0, 0), (7, 1), (23, 2)]
    g = gradref.gradient(v, f, 1, ta, picks)
    h = 1e-4
    for k, (vv, c) in enumerate(picks):
        vp, vm = v.copy(), v.copy()
        vp[vv, c] += h
        vm[vv, c] -= h
        fp = ob.best_run(meshes.to_triangles(vp, f), ta, tv, iarea=1, ivisco=1)
        fm = ob.best_run(meshes.to_triangles(vm, f), ta, tv, iarea=1, ivisco=1)
        fd = np.array([fp.report["DTRANS"] - fm.report["DTRANS"], fp.report["DR"] - fm.report["DR"],
                       fp.chiprime - fm.chiprime]) / (2 * h)
        assert np.all(np.abs(fd - g[:, k]) <= 1e-6 * np.abs(g[:, k]) + 1e-9 * np.abs(fd).max()), (fd, g[:, k])
