"""CPU tests of the product's C++ host driver (include/best_driver.h) against the oracle's numpy
restatement of the same Fortran: two independent restatements of best.f's set-up, COMPON, the
deflation vectors, DIFCO, VISCO and OUTPUT's traces, fed with the oracle's LAPACK solutions."""
import numpy as np
import pytest

import best_hydro_b200 as bh
from oracle import best as ob
from tests.helpers import golden_mesh


@pytest.fixture(scope="module", params=["2eu7_02562", "1aki49_atom_01806"])
def case(request):
    tri, ta, tv = golden_mesh(request.param)
    o = ob.best_run(tri, ta, tv, iarea=1, ivisco=1, icov=1, wm=30000.0)
    return tri, ta, tv, o


def test_setup_compon_deflation_bitwise(case):
    tri, ta, tv, o = case
    s = bh.Setup(tri, 1, ta)
    v1, v2, v3 = o.setup.colmajor()
    for a, b in ((s.v1, v1), (s.v2, v2), (s.v3, v3), (s.area, o.setup.area)):
        assert np.array_equal(a, b)
    assert s.afac == o.setup.afac and s.totarea == o.setup.totarea
    assert (s.ncomp, s.nopen, s.ndef) == (o.setup.ncomp, o.setup.nopen, o.setup.ndef)
    assert np.array_equal(s.icomp, o.setup.icomp)
    xmu, gdef = s.deflation(o.diagm)
    assert np.array_equal(xmu, o.xmu)
    np.testing.assert_array_equal(gdef, o.gdef)


def test_rhs_and_postprocessing(case):
    tri, ta, tv, o = case
    assert np.array_equal(bh.rhs6(o.x), ob.rhs6(o.x, o.setup.n))
    assert np.array_equal(bh.strain5(o.x), ob.strain5(o.x, o.setup.n))
    t = bh.difco(o.x, o.setup.area, o.B6)
    for k in ("Dtt", "Dtr", "Drr", "urc", "udr"):
        np.testing.assert_allclose(t[k], o.tensors[k], rtol=1e-13, atol=1e-13 * np.max(np.abs(o.tensors[k])))
    chip, dv = bh.visco(o.x, o.setup.area, o.V5, o.B6, icov=1)
    assert abs(chip / o.chiprime - 1) < 1e-13
    np.testing.assert_allclose(dv, o.dvisc, rtol=1e-12)
    tr = bh.traces(t)
    assert abs(tr["DTRANS"] / o.report["DTRANS"] - 1) < 1e-13
    assert abs(tr["DR"] / o.report["DR"] - 1) < 1e-13


def test_extrapolation_in_one_over_n():
    """bgpu_best_extrapolate: least squares of y on 1/N, exact on a line, equal to numpy's fit."""
    n = [2420, 2880, 3920, 5120, 6480, 8000, 9680, 10580]
    y = [1.5 - 7.0 / k for k in n]
    y0, slope = bh.extrapolate(n, y)
    assert abs(y0 - 1.5) < 1e-13 and abs(slope + 7.0) < 1e-9
    rng = np.random.default_rng(3)
    y = 1.0 + 50.0 / np.array(n) + 1e-6 * rng.standard_normal(len(n))
    s_np, y_np = np.polyfit(1.0 / np.array(n, dtype=float), y, 1)
    y0, slope = bh.extrapolate(n, y)
    assert abs(y0 - y_np) < 1e-12 and abs(slope - s_np) < 1e-6 * abs(s_np)
