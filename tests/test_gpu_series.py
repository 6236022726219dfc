"""A series of meshes solved together (include/best_gpu.h, bgpu_series_*): one assembly launch for
every mesh, each step of the FP64 LU batched over the meshes, the whole build replayed from one CUDA
graph.  Each mesh's solution must be the one the single-mesh plain path gives (bhm_build with
direct = 1), bit for bit: the batch changes which CTA computes what, never the arithmetic."""
import numpy as np
import pytest

import best_hydro_b200 as bh
from best_hydro_b200 import meshes
from tests.helpers import golden_mesh

pytestmark = pytest.mark.gpu


def single_solve(st, rhs):
    s = bh.BhmSolver()
    s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = s.incenters()
    xmu, gdef = st.deflation(s.diag_mean())
    bh.set_precision(bh.BGPU_FP64)
    s.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
    out = s.solve(rhs)
    s.destroy()
    bh.set_precision(-1)
    return x, out


def ellipsoid_setups(freqs):
    out = []
    for f in freqs:
        tri, ta, tv = meshes.ellipsoid(f)
        out.append(bh.Setup(tri, 1, ta))
    return out


@pytest.mark.parametrize("tune", [0, 1])
def test_series_equals_single_solves(tune):
    # orders 960, 1500, 2160, 3840: last block columns of 192, 220, 112 and 256 (a whole one)
    setups = ellipsoid_setups([4, 5, 6, 8])
    tri, ta, tv = golden_mesh("1aki49_atom_01806")  # two surfaces: per-mesh deflation offsets
    setups.append(bh.Setup(tri, 0, ta))
    per, ext, tm = bh.series_run(setups, tune=tune)
    print(f"\nseries build {tm['build']:.1f} ms (assembly {tm['assemble']:.1f}), solve {tm['solve']:.1f} ms, "
          f"tuning pass {tm['tune']:.1f} ms")
    for st, d in zip(setups, per):
        s = bh.BhmSolver()
        s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        x = s.incenters()
        s.destroy()
        rhs = np.hstack([bh.rhs6(x), bh.strain5(x)])
        x1, sol = single_solve(st, rhs)
        assert np.array_equal(sol.view(np.int64), d["solution"].view(np.int64)), f"N={st.n}"
    if tune:
        table = bh.autotune_table()
        print("\n".join(table))
        assert table


def test_series_extrapolates_like_numpy():
    setups = ellipsoid_setups([4, 5, 6])
    per, ext, _ = bh.series_run(setups)
    n = np.array([d["N"] for d in per], dtype=float)
    for key in ("D_t", "D_r", "chiprime"):
        y = np.array([d[key] for d in per])
        slope, y0 = np.polyfit(1.0 / n, y, 1)
        assert abs(ext[key] - y0) <= 1e-12 * abs(y0), key


def test_series_rejects_bad_input():
    n = np.zeros(1, dtype=np.int32)
    z = np.zeros(1)
    assert bh.lib().bgpu_series_create(0, n.ctypes.data_as(bh._ip), bh._p(z), bh._p(z), bh._p(z), bh._p(z), bh._p(z),
                                       1.0) != 0
    assert bh.lib().bgpu_series_create(1, n.ctypes.data_as(bh._ip), bh._p(z), bh._p(z), bh._p(z), bh._p(z), bh._p(z),
                                       1.0) != 0  # a mesh without triangles
    bh.lib().bgpu_series_destroy()
    with pytest.raises(bh.BestGpuError):
        bh.Series().solve([np.zeros((3, 1))])
    bh.log_lines()
