"""GPU records of the workloads at their full sizes (the ellipsoid 30/20/12 A, geodesic frequency 16,
N = 5,120, normal jitter U(+-2%) seed 0; its series at the eight frequencies 11 .. 23; the star body
at frequency 45, N = 40,500):

  * ellipsoid N = 5,120: every GR entry bit for bit TGETGR's arithmetic with correctly rounded
    functions; D_t, D_r, D_tr, centres and CHI' within 1e-10 of the oracle (FP64 path) and 1e-8
    (mixed path); without the jitter, D_t and D_r within the discretisation error of Perrin's
    analytic ellipsoid (0.2 % and 0.5 % at this N, oracle/perrin.py);
  * the series f = 11, 12, 14, 16, 18, 20, 22, 23 (N = 2,420 .. 10,580): each mesh's solution bit
    for bit its single-mesh FP64 solve, the 1/N extrapolation as numpy's;
  * adjoint gradients at N = 5,120 against central differences (h = 1e-4 A) on 12 random vertices
    (seed 2);
  * star body N = 40,500 (order 121,500): the mixed path within 1e-8 of the FP64 path, which needs
    118 GB (a B200 holds it; the mixed path then copies its operands per product, as its BF16
    mirrors do not fit beside the FP64 matrix).
"""
import numpy as np
import pytest

import best_hydro_b200 as bh
from best_hydro_b200 import meshes
from oracle import best as ob
from oracle import perrin
from tests import crshim
from tests.helpers import rel, run_gpu

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _compare(g, o, tol):
    for key in ("Dtt", "Drr"):
        assert rel(g["tensors"][key], o.tensors[key]) < tol, key
    scale = np.sqrt(np.max(np.abs(o.tensors["Dtt"])) * np.max(np.abs(o.tensors["Drr"])))
    assert np.max(np.abs(g["tensors"]["Dtr"] - o.tensors["Dtr"])) / scale < tol
    size = np.sqrt(np.mean(o.x.reshape(3, -1) ** 2) * 3)
    for key in ("urc", "udr"):
        assert np.max(np.abs(g["tensors"][key] - o.tensors[key])) / size < tol, key
    assert abs(g["chiprime"] / o.chiprime - 1) < tol


def test_ellipsoid_5120_entries_are_correctly_rounded_tgetgr():
    torch = _torch()
    tri, ta, tv = meshes.ellipsoid(16)
    s = ob.setup(tri, 1, ta)
    solver = bh.BhmSolver()
    v1, v2, v3 = s.colmajor()
    solver.create(v1, v2, v3, s.area, s.afac, 1.0)
    n3 = 3 * s.n
    d = torch.empty((n3, n3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    bh.assemble_device(0, s.n, 0, s.n, d.data_ptr(), n3)
    torch.cuda.synchronize()
    got = d.cpu().numpy()  # row j = column j of GR
    del d
    cr, x, _ = crshim.assemble_cr(s, 1.0)
    ndiff = int(np.count_nonzero(got.view(np.int64) != cr.T.view(np.int64)))
    print(f"\nN={s.n}: {ndiff} of {got.size} entries differ from the correctly rounded evaluation")
    assert ndiff == 0
    assert np.array_equal(solver.incenters().view(np.int64), x.view(np.int64))
    solver.destroy()


@pytest.mark.parametrize("direct,tol", [(1, 1e-10), (0, 1e-8)])
def test_ellipsoid_5120_vs_oracle(direct, tol):
    tri, ta, tv = meshes.ellipsoid(16)
    o = ob.best_run(tri, ta, tv, iarea=1, ivisco=1)
    g = run_gpu(bh.BhmSolver(), tri, ta, iarea=1, direct=direct, eps=1e-10, ivisco=1)
    _compare(g, o, tol)


@pytest.mark.parametrize("direct", [1, 0])
def test_ellipsoid_5120_vs_perrin(direct):
    DT, DR, _, _ = perrin.perrin((30.0, 20.0, 12.0))
    tri, ta, tv = meshes.ellipsoid(16, jitter=0.0)
    g = run_gpu(bh.BhmSolver(), tri, ta, iarea=1, direct=direct, eps=1e-10)
    et, er = g["report"]["DTRANS"] / DT - 1, g["report"]["DR"] / DR - 1
    print(f"\nN=5120 against Perrin: D_t {et:+.2e}, D_r {er:+.2e}")
    assert 0 < et < 2e-3 and 0 < er < 5e-3


def test_series_at_the_eight_frequencies():
    freqs = (11, 12, 14, 16, 18, 20, 22, 23)
    setups = []
    for f in freqs:
        tri, ta, tv = meshes.ellipsoid(f)
        setups.append(bh.Setup(tri, 1, ta))
    per, ext, tm = bh.series_run(setups, tune=1)
    print(f"\nseries N={[st.n for st in setups]}: build {tm['build']:.1f} ms (assembly {tm['assemble']:.1f}), "
          f"solve {tm['solve']:.1f} ms")
    bh.set_precision(bh.BGPU_FP64)
    try:
        for st, d in zip(setups, per):
            s = bh.BhmSolver()
            s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
            x = s.incenters()
            xmu, gdef = st.deflation(s.diag_mean())
            s.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
            sol = s.solve(np.hstack([bh.rhs6(x), bh.strain5(x)]))
            s.destroy()
            assert np.array_equal(sol.view(np.int64), d["solution"].view(np.int64)), f"N={st.n}"
    finally:
        bh.set_precision(-1)
    n = np.array([d["N"] for d in per], dtype=float)
    for key in ("D_t", "D_r", "chiprime"):
        y = np.array([d[key] for d in per])
        slope, y0 = np.polyfit(1.0 / n, y, 1)
        assert abs(ext[key] - y0) <= 1e-12 * abs(y0), key


def test_mixed_series_at_the_eight_frequencies():
    """The series with every mesh's factorisation on the tensor cores (one stream per mesh, all
    enqueued together) and FP64 GMRES-IR: each mesh's D_t, D_r, CHI' within 1e-8 of its plain FP64
    solve, and the 1/N extrapolation likewise."""
    freqs = (11, 12, 14, 16, 18, 20, 22, 23)
    setups = []
    for f in freqs:
        tri, ta, tv = meshes.ellipsoid(f)
        setups.append(bh.Setup(tri, 1, ta))
    per64, ext64, _ = bh.series_run(setups)
    perm, extm, tm = bh.series_run(setups, precision=bh.BGPU_MIXED)
    print(f"\nmixed series build {tm['build']:.1f} ms, solve {tm['solve']:.1f} ms")
    assert any("mixed precision" in ln for ln in bh.log_lines())
    for a, b in zip(perm, per64):
        for key in ("D_t", "D_r", "chiprime"):
            assert abs(a[key] / b[key] - 1) < 1e-8, (a["N"], key)
    for key in ("D_t", "D_r", "chiprime"):
        assert abs(extm[key] / ext64[key] - 1) < 1e-8, key


def test_adjoint_at_5120():
    verts, faces, ta, tv = meshes.ellipsoid_vf(16)
    from tests.test_gpu_adjoint import check_fd
    rng = np.random.default_rng(2)
    check_fd(verts, faces, ta, 1, rng.choice(len(verts), 12, replace=False))


def test_star_40500_mixed_vs_fp64():
    tri, ta, tv = meshes.star(45)
    st = bh.Setup(tri, 0, ta)
    s = bh.BhmSolver()
    s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = s.incenters()
    xmu, gdef = st.deflation(s.diag_mean())
    rhs = np.hstack([bh.rhs6(x), bh.strain5(x)])
    out = {}
    for prec in (bh.BGPU_FP64, bh.BGPU_MIXED):
        bh.set_precision(prec)
        s.build(eps=1e-10, direct=1 if prec == bh.BGPU_FP64 else 0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        B = s.solve(rhs)
        t = bh.difco(x, st.area, B[:, :6])
        chip, _ = bh.visco(x, st.area, B[:, 6:], B[:, :6])
        tr = bh.traces(t)
        out[prec] = (tr["DTRANS"], tr["DR"], chip, t)
        print(f"\n{'fp64' if prec == bh.BGPU_FP64 else 'mixed'}: {bh.timings()}")
    bh.set_precision(-1)
    s.destroy()
    a, b = out[bh.BGPU_MIXED], out[bh.BGPU_FP64]
    for i in range(3):
        assert abs(a[i] / b[i] - 1) < 1e-8, i
    for key in ("Dtt", "Drr"):
        assert rel(a[3][key], b[3][key]) < 1e-8, key
