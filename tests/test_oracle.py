"""CPU tests of the oracle: the C restatement of TGETGR/triangleint against the reference's own
kernel.cpp (bit for bit) and the committed golden sample; the whole numpy/OpenBLAS restatement
against the reference's golden end results (test/expected_best_*.txt at their 2e-4)."""
import numpy as np
import pytest

from oracle import best as ob
from best_hydro_b200 import meshes
from tests.helpers import expected_cases, golden_mesh, value_for_label


def test_c_restatement_matches_golden_sample():
    """Entries, incenters and DIAGM of 2eu7_02562 from the reference's kernel.cpp (committed
    fixture) are reproduced bit for bit by the C restatement."""
    g = np.load(f"{ob.HERE}/../tests/golden/gr_2eu7_sample.npz")
    tri, ta, tv = golden_mesh("2eu7_02562")
    s = ob.setup(tri, 1, ta)
    gr, x, self9 = ob.assemble(s)
    assert np.array_equal(gr[:96, :96].view(np.int64), g["corner"].view(np.int64))
    assert np.array_equal(gr[g["ii"], g["jj"]].view(np.int64), g["vals"].view(np.int64))
    assert np.array_equal(x.view(np.int64), g["x"].view(np.int64))
    assert ob.diag_mean(self9, s.n) == float(g["diag_mean"])


@pytest.mark.skipif(ob.ref_lib() is None, reason="oracle/_ref (the reference's kernel.cpp) not built")
@pytest.mark.parametrize("case", ["icosphere", "ellipsoid_f6", "two_surface_pm"])
def test_c_restatement_bit_exact_vs_reference(case):
    if case == "icosphere":
        tri, ta, tv = meshes.icosphere(2, 20.0)
        s = ob.setup(tri, 1, ta)
        cg = 1.0
    elif case == "ellipsoid_f6":
        tri, ta, tv = meshes.ellipsoid(6)
        s = ob.setup(tri, 0, None)
        cg = 1.0
    else:
        tri, ta, tv = golden_mesh("1aki49_atom_01806")
        s = ob.setup(tri, 1, ta)
        cg = 0.0  # -p (pre-averaged) as well
    gr, x, self9 = ob.assemble(s, cg)
    r = ob.assemble_ref(s, cg)
    h, worst = ob.ulp_hist(gr, r[0])
    assert worst == 0, h
    assert np.array_equal(x.view(np.int64), r[1].view(np.int64))
    assert ob.diag_mean(self9, s.n) == r[2]


@pytest.mark.parametrize("key", ["2eu7", "2eu7_vc", "2eu7_na", "two"])
def test_oracle_reproduces_reference_golden_results(key):
    c = expected_cases()[key]
    tri, ta, tv = golden_mesh(c["mesh"])
    res = ob.best_run(tri, ta, tv, iarea=c["iarea"], ivisco=c["ivisco"], icov=c["icov"], wm=c["wm"])
    for e in c["expected"]:
        want = e["value"]
        if e["label"] in ("Dx", "Dy", "Dz"):
            got = res.dvisc["xyz".index(e["label"][1])]
        else:
            got = value_for_label(res.report, e["label"])
        assert abs(got - want) <= e["tol"] * abs(want), (e["label"], got, want)
    if key == "two":
        assert res.setup.ncomp == 2 and res.setup.nopen == 0 and res.setup.ndef == 2


def test_frame_permutation_invariance():
    """check_best_frame.pl's property: cyclically permuting the axes permutes the tensors."""
    tri, ta, tv = meshes.ellipsoid(5)
    r1 = ob.best_run(tri, ta, tv, iarea=1)
    perm = np.concatenate([[3 * k + 1, 3 * k + 2, 3 * k] for k in range(3)])
    r2 = ob.best_run(tri[:, perm], ta, tv, iarea=1)
    P = np.array([[0, 1, 0], [0, 0, 1], [1, 0, 0]], dtype=float)
    for key in ("Dtt", "Drr"):
        np.testing.assert_allclose(P @ r1.tensors[key] @ P.T, r2.tensors[key], rtol=1e-9, atol=1e-12)


def test_sphere_limits():
    """Stokes sphere: D_t -> 4/(3R), D_r -> 1/R^3 (internal units) as N grows."""
    R = 20.0
    tri, ta, tv = meshes.icosphere(3, R)
    r = ob.best_run(tri, ta, tv, iarea=1)
    assert abs(r.report["trace_dtt"] * 3 * R / 4 - 1) < 5e-3
    assert abs(r.report["trace_drr"] * R ** 3 - 1) < 2e-2


def test_mesh_generators_sizes_and_closure():
    for f in (11, 16):
        tri, _, _ = meshes.ellipsoid(f)
        assert tri.shape == (20 * f * f, 9)
        s = ob.setup(tri, 0, None)
        assert s.nopen == 0 and s.ncomp == 1
    tri, ta, _ = meshes.icosphere(3, 20.0)
    assert tri.shape == (1280, 9)
    tri, _, _ = meshes.star(8)
    assert tri.shape == (1280, 9)
    s = ob.setup(tri, 0, None)
    assert s.nopen == 0


def test_compon_open_surface_falls_back_to_one_deflation():
    """compon.f90 + best.f:325-332: an open surface gets one deflation term (NDEF = 1)."""
    tri, ta, tv = meshes.icosphere(1, 10.0)
    s = ob.setup(tri[1:], 0, None)
    assert s.nopen > 0 and s.ndef == 1 and np.all(s.icomp == 1)


def test_self_blocks_differ_from_glibc_only_where_glibc_misrounds():
    """The reference's self-block arithmetic with correctly rounded acos/sin/cos/log (what the GPU
    kernel computes) against the same arithmetic with glibc's: the few entries that differ are within
    4 ulp of their block's largest entry (cancellation residues of glibc's misrounded calls)."""
    from tests import crshim
    tri, ta, tv = golden_mesh("2eu7_02562")
    s = ob.setup(tri, 1, ta)
    x_cr, s_cr = crshim.self_blocks_cr(s)
    x_g, s_g = ob.incenters_and_self(s)
    assert np.array_equal(x_cr, x_g)  # incenters use no transcendental function
    same = np.count_nonzero(s_cr == s_g)
    assert same >= 0.99 * s_g.size
    assert np.max(crshim.block_scale_ulps(s_cr, s_g)) <= 4


def test_pair_blocks_long_double():
    """The long-double pair blocks (the reference value the mixed assembly is compared with) agree
    with the FP64 restatement within the FP64 formula's own error: 1e-10 of the row scale."""
    tri, ta, tv = golden_mesh("2eu7_02562")
    s = ob.setup(tri, 1, ta)
    x, _ = ob.incenters_and_self(s, 1.0)
    gr, _, _ = ob.assemble(s, 1.0, rows=(0, 40), cols=(0, s.n))
    rng = np.random.default_rng(3)
    rows = rng.integers(0, 40, 200)
    cols = rng.integers(0, s.n, 200)
    keep = rows != cols
    rows, cols = rows[keep], cols[keep]
    t = ob.pair_blocks_ld(s, x, rows, cols, 1.0)
    scale = np.abs(gr).reshape(40, 3, -1).max(axis=(1, 2))
    for k, (r, c) in enumerate(zip(rows, cols)):
        g = gr[3 * r:3 * r + 3, 3 * c:3 * c + 3]
        assert np.abs(g - t[k]).max() / scale[r] < 1e-10
