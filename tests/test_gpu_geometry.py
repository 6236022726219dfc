"""GPU parity of BEST's input set-up done on the device (bgpu_create_from_triangles,
bgpu_build_prepared): centroid shift, areas and the area correction (best/best.f:261-315), COMPON's
surfaces and open edges (best/compon.f90:19-116), NDEF (best.f:323-337), XMU and GDEF
(best.f:384-404, DEFGAM compon.f90:185-197).  Every array and scalar must equal the host
restatement's (bgpu_best_setup, bgpu_best_deflation; pinned to the oracle by tests/test_driver.py)
bit for bit, and the solve built from them must equal the solve built from the host's arrays bit for
bit.  Meshes: one surface with the area correction, two surfaces (1aki49), the mesh's own area
(ellipsoid), an open surface (a half sphere: open edges, so NDEF = 1)."""
import numpy as np
import pytest

import best_hydro_b200 as bh
from best_hydro_b200 import meshes
from tests.helpers import golden_mesh

pytestmark = pytest.mark.gpu


def _half_sphere():
    tri, ta, tv = meshes.icosphere(3, 20.0)
    cz = (tri[:, 2] + tri[:, 5] + tri[:, 8]) / 3
    return tri[cz > 0], None, None


CASES = {
    "2eu7_02562": lambda: (golden_mesh("2eu7_02562"), 1),
    "1aki49_two_surfaces": lambda: (golden_mesh("1aki49_atom_01806"), 1),
    "ellipsoid_f12_na": lambda: (meshes.ellipsoid(12), 0),
    "half_sphere_open": lambda: (_half_sphere(), 0),
}


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes(order="F") == b.tobytes(order="F")


@pytest.mark.parametrize("case", list(CASES))
def test_device_setup_equals_host_setup(case):
    (tri, ta, tv), iarea = CASES[case]()
    tri = np.ascontiguousarray(tri, dtype=np.float64)
    st = bh.Setup(tri, iarea, ta)
    if case == "half_sphere_open":
        assert st.nopen > 0 and st.ndef == 1
    if case == "1aki49_two_surfaces":
        assert st.ndef == 2
    s = bh.BhmSolver()
    info, counts = s.create_from_triangles(tri, iarea, ta)
    assert (counts["ncomp"], counts["nopen"], counts["ndef"]) == (st.ncomp, st.nopen, st.ndef)
    assert info["afac"] == st.afac and info["totarea"] == st.totarea
    assert _same(info["centroid"], st.centroid)
    x_dev, dm_dev = s.incenters(), s.diag_mean()
    s.build_prepared(eps=1e-10, direct=1)
    v1, v2, v3, area, icomp, xmu, gdef = s.prepared_arrays(st.ndef)
    for got, want in ((v1, st.v1), (v2, st.v2), (v3, st.v3), (area, st.area)):
        assert _same(got, want)
    if st.ndef > 1 or st.nopen > 0:
        assert np.array_equal(icomp, st.icomp)
    xmu_h, gdef_h = st.deflation(dm_dev)
    assert _same(xmu, xmu_h) and _same(gdef, gdef_h)
    B_dev = s.solve(bh.rhs6(x_dev))
    s.destroy()
    # the same solve from the host's arrays through bhm_create / bhm_build
    s2 = bh.BhmSolver()
    s2.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = s2.incenters()
    assert _same(x, x_dev) and s2.diag_mean() == dm_dev
    s2.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef_h, comp=st.icomp, xmu=xmu_h)
    B = s2.solve(bh.rhs6(x))
    s2.destroy()
    assert _same(B_dev, B)
