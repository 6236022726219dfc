"""GPU tests of the H-matrix path (bgpu_set_precision(BGPU_HMATRIX); the GPU counterpart of the
reference's H-matrix solver, hmatrix/src/api.cpp:582-771, which BEST runs for large N):

* its product (H + deflation) x against the dense deflated GR (bhm_entries + best.f:406-425) at
  eps = 1e-4 and 1e-6: relative error per column <= 3 eps;
* BEST's results (D_t, D_r, D_tr, centres, CHI') from its GMRES solves against the plain FP64 path on
  the same mesh: relative difference <= eps;
* the reference's golden results of 2eu7 (one surface, area correction) and of the two-surface case
  (NDEF = 2, the deflation per surface) within their 2e-4 tolerance, as the reference's H-matrix
  path meets them (test/run_tests.sh).
"""
import numpy as np
import pytest
import torch

import best_hydro_b200 as bh
from best_hydro_b200 import BhmSolver, meshes
from oracle import best as ob
from tests.helpers import expected_cases, golden_mesh, rel, run_gpu, value_for_label

pytestmark = pytest.mark.gpu


def _run(tri, ta, precision, eps=1e-4, ivisco=1, **kw):
    bh.set_precision(precision)
    solver = BhmSolver()
    try:
        g = run_gpu(solver, tri, ta, eps=eps, direct=1 if precision == bh.BGPU_FP64 else 0, ivisco=ivisco, **kw)
        g["stats"] = bh.hmatrix_stats() if precision == bh.BGPU_HMATRIX else None
        g["precision"] = bh.lib().bgpu_precision()
    finally:
        bh.set_precision(-1)
    return solver, g


def _results_diff(a, b):
    ta, tb = a["tensors"], b["tensors"]
    out = {k: rel(ta[k], tb[k]) for k in ("Dtt", "Drr")}
    scale = np.sqrt(np.max(np.abs(tb["Dtt"])) * np.max(np.abs(tb["Drr"])))
    out["Dtr"] = float(np.max(np.abs(ta["Dtr"] - tb["Dtr"])) / scale)
    size = np.sqrt(np.mean(b["x"].reshape(3, -1) ** 2) * 3)
    for k in ("urc", "udr"):
        out[k] = float(np.max(np.abs(ta[k] - tb[k])) / size)
    if a.get("chiprime") is not None:
        out["chiprime"] = abs(a["chiprime"] / b["chiprime"] - 1)
    return out


@pytest.mark.parametrize("eps", [1e-4, 1e-6])
def test_product_against_dense(eps):
    tri, ta, tv = meshes.ellipsoid(12)  # N = 2,880
    solver, g = _run(tri, ta, bh.BGPU_HMATRIX, eps=eps, ivisco=0)
    assert g["precision"] == bh.BGPU_HMATRIX
    s = g["setup"]
    n3 = 3 * s.n
    gr = solver.entries(0, n3, 0, n3)
    ob.deflate(s, gr, g["xmu"], g["gdef"])
    rng = np.random.default_rng(7)
    X = np.asfortranarray(rng.standard_normal((n3, 3)))
    Y = gr @ X
    dx = torch.from_numpy(X.T.copy()).cuda()  # column-major 3n x 3: row c of the torch tensor is column c
    dy = torch.zeros_like(dx)
    bh.hmatrix_matvec_device(3, dx.data_ptr(), n3, dy.data_ptr(), n3)
    torch.cuda.synchronize()
    Yh = dy.cpu().numpy().T
    err = np.linalg.norm(Yh - Y, axis=0) / np.linalg.norm(Y, axis=0)
    st = g["stats"]
    print(f"eps {eps}: product error {err.max():.2e}; {st}")
    assert st["lowrank_blocks"] > 0 and st["dense_blocks"] > 0
    assert st["dense_entries"] + st["lowrank_entries"] < 0.9 * n3 * n3
    assert err.max() <= 3 * eps, err
    solver.destroy()


@pytest.mark.parametrize("eps", [1e-4, 1e-6])
def test_results_against_fp64_path(eps):
    tri, ta, tv = meshes.ellipsoid(16)  # N = 5,120
    s1, h = _run(tri, ta, bh.BGPU_HMATRIX, eps=eps)
    s1.destroy()
    s2, d = _run(tri, ta, bh.BGPU_FP64)
    s2.destroy()
    diff = _results_diff(h, d)
    print(f"eps {eps}: {diff}; GMRES steps {h['stats']['gmres_steps']:.0f}; {h['stats']}")
    assert h["stats"]["relres"] <= 0.1 * eps
    for k, v in diff.items():
        assert v <= eps, (k, v)


@pytest.mark.parametrize("key", ["2eu7", "two"])
def test_golden_results_on_the_hmatrix(key):
    c = expected_cases()[key]
    tri, ta, tv = golden_mesh(c["mesh"])
    solver, g = _run(tri, ta, bh.BGPU_HMATRIX, eps=1e-4, ivisco=c["ivisco"], iarea=c["iarea"], icov=c["icov"],
                     truevol=tv, wm=c["wm"])
    for e in c["expected"]:
        if e["label"] in ("Dx", "Dy", "Dz"):
            got = g["dvisc"]["xyz".index(e["label"][1])]
        else:
            got = value_for_label(g["report"], e["label"])
        assert abs(got - e["value"]) <= e["tol"] * abs(e["value"]), (e["label"], got, e["value"])
    solver.destroy()


def test_product_at_the_headline_size():
    """The star body at N = 20,480 (the benchmark's mesh; trees of depth 8, blocks up to 10,240
    triangles a side) at eps = 1e-6: the product against the dense deflated GR, formed in row blocks
    by the exact assembly, within 3 eps; no block row is missed."""
    tri, ta, tv = meshes.star(32)
    st = bh.Setup(tri, 0, ta)
    s = BhmSolver()
    s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = s.incenters()
    xmu, gdef = st.deflation(s.diag_mean())
    n = st.n
    n3 = 3 * n
    bh.set_precision(bh.BGPU_HMATRIX)
    try:
        s.build(eps=1e-6, direct=0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
    finally:
        bh.set_precision(-1)
    rng = np.random.default_rng(3)
    X = rng.standard_normal((n3, 2))
    dx = torch.from_numpy(X.T.copy()).cuda()
    dy = torch.zeros_like(dx)
    bh.hmatrix_matvec_device(2, dx.data_ptr(), n3, dy.data_ptr(), n3)
    torch.cuda.synchronize()
    Yh = dy.cpu().numpy().T
    Y = np.zeros((n3, 2))
    for r0 in range(0, n, 2048):
        r1 = min(n, r0 + 2048)
        blk = torch.empty((n3, 3 * (r1 - r0)), dtype=torch.float64, device="cuda")  # rows of r0..r1, column-major
        bh.assemble_device(r0, r1, 0, n, blk.data_ptr(), 3 * (r1 - r0))
        Y[3 * r0:3 * r1] = (dx @ blk).cpu().numpy().T
        del blk
    torch.cuda.empty_cache()  # later tests size their paths by the device's free memory
    xm = xmu.reshape(-1)
    Y += np.outer(xm, gdef[0] * (xm @ X))  # one surface
    err = np.linalg.norm(Yh - Y, axis=0) / np.linalg.norm(Y, axis=0)
    rows = np.abs(Yh - Y).max(axis=1) / (np.linalg.norm(Y) / np.sqrt(n3))
    print(f"N={n}: product error {err.max():.2e}, worst row {rows.max():.2e}; {bh.hmatrix_stats()}")
    assert st.ndef == 1
    assert err.max() <= 3e-6, err
    assert rows.max() <= 1e-3
    s.destroy()


def test_device_setup_path_and_determinism():
    """The H-matrix path behind the device set-up (bgpu_create_from_triangles + bgpu_build_prepared)
    on the two-surface mesh (NDEF = 2) gives, bit for bit, the solution of the host path (bhm_create +
    bhm_build with the host's arrays): the set-up's arrays are equal, and the H-matrix build and its
    GMRES solve are deterministic (fixed summation orders, no atomics)."""
    tri, ta, tv = golden_mesh(expected_cases()["two"]["mesh"])
    tri = np.ascontiguousarray(tri, dtype=np.float64)
    st = bh.Setup(tri, 1, ta)
    assert st.ndef == 2
    bh.set_precision(bh.BGPU_HMATRIX)
    try:
        s = BhmSolver()
        s.create_from_triangles(tri, 1, ta)
        x_dev, dm_dev = s.incenters(), s.diag_mean()
        s.build_prepared(eps=1e-5, direct=0)
        assert bh.lib().bgpu_precision() == bh.BGPU_HMATRIX
        B_dev = s.solve(bh.rhs6(x_dev))
        s.destroy()
        s2 = BhmSolver()
        s2.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        x = s2.incenters()
        xmu, gdef = st.deflation(s2.diag_mean())
        s2.build(eps=1e-5, direct=0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        B = s2.solve(bh.rhs6(x))
        s2.destroy()
    finally:
        bh.set_precision(-1)
    assert np.array_equal(x, x_dev)
    assert np.array_equal(B, B_dev)


@pytest.mark.parametrize("precision", [-1, bh.BGPU_HMATRIX])
def test_whole_program_on_golden_mesh(tmp_path, precision):
    """BEST's whole program through the seam (bgpu_best_run, the best_gpu command; -hm selects the
    H-matrix path) on 2eu7 with -v and a molecular weight: the reference's golden values within their
    tolerance, and the .be and .log files written."""
    c = expected_cases()["2eu7"]
    tri, ta, tv = golden_mesh(c["mesh"])
    path = tmp_path / "2eu7.txt"
    meshes.write_best(str(path), tri, ta, tv)
    bh.log_lines()  # the program's .log takes the library's queued messages: start from an empty queue
    rep = bh.best_run(path, iarea=c["iarea"], ivisco=c["ivisco"], icov=c["icov"], wm=c["wm"], precision=precision)
    bh.set_precision(-1)
    for e in c["expected"]:
        if e["label"] in ("Dx", "Dy", "Dz"):
            got = rep["dvisc"]["xyz".index(e["label"][1])]
        else:
            got = value_for_label(rep, e["label"])
        assert got is not None, e["label"]
        assert abs(got - e["value"]) <= e["tol"] * abs(e["value"]), (e["label"], got, e["value"])
    outs = sorted(p.name for p in tmp_path.iterdir())
    assert any(n.endswith(".be") for n in outs) and any(n.endswith(".log") for n in outs), outs
    log = "".join(p.read_text() for p in tmp_path.iterdir() if p.name.endswith(".log"))
    assert ("GPU build: H-matrix of order 7686" in log) == (precision == bh.BGPU_HMATRIX), log[-2000:]
