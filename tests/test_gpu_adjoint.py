"""The adjoint gradients of D_t, D_r and [eta] (include/best_gpu.h, bgpu_best_gradient) against
central finite differences of the whole GPU pipeline (set-up, assembly, deflation, FP64 LU, the 11
solves, DIFCO/VISCO/OUTPUT), on shared vertices, h = 1e-4 A."""
import numpy as np
import pytest

import best_hydro_b200 as bh
from best_hydro_b200 import meshes
from tests.helpers import golden_mesh

pytestmark = pytest.mark.gpu
H = 1e-4


def values_of(tri, ta, iarea):
    """BEST's D_t, D_r and CHI' through the seam with the FP64 LU."""
    st = bh.Setup(tri, iarea, ta)
    s = bh.BhmSolver()
    s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = s.incenters()
    xmu, gdef = st.deflation(s.diag_mean())
    bh.set_precision(bh.BGPU_FP64)
    s.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
    B = s.solve(np.hstack([bh.rhs6(x), bh.strain5(x)]))
    tr = bh.traces(bh.difco(x, st.area, B[:, :6]))
    chip, _ = bh.visco(x, st.area, B[:, 6:], B[:, :6])
    return np.array([tr["DTRANS"], tr["DR"], chip]), s, st


def check_fd(verts, faces, ta, iarea, picks):
    tri = meshes.to_triangles(verts, faces)
    v0, s, st = values_of(tri, ta, iarea)
    vals, g = s.gradient(iarea=iarea, truearea=ta or 0.0)
    bh.set_precision(-1)
    assert np.allclose(vals, v0, rtol=1e-13, atol=0), (vals, v0)
    gv = meshes.corner_to_vertex(g, faces, len(verts))  # (3 results, vertices, 3)
    worst = np.zeros(3)
    for v in picks:
        for c in range(3):
            vp, vm = verts.copy(), verts.copy()
            vp[v, c] += H
            vm[v, c] -= H
            fp = values_of(meshes.to_triangles(vp, faces), ta, iarea)[0]
            fm = values_of(meshes.to_triangles(vm, faces), ta, iarea)[0]
            fd = (fp - fm) / (2 * H)
            err = np.abs(fd - gv[:, v, c]) / np.abs(gv).reshape(3, -1).max(axis=1)
            worst = np.maximum(worst, err)
    bh.set_precision(-1)
    print(f"\nN={len(faces)} iarea={iarea} ndef={st.ndef}: worst |FD - adjoint| / max|grad| "
          f"D_t {worst[0]:.2e}, D_r {worst[1]:.2e}, CHI' {worst[2]:.2e}")
    assert np.all(worst < 1e-6), worst
    return gv


def test_adjoint_ellipsoid_with_area_correction():
    verts, faces, ta, tv = meshes.ellipsoid_vf(6)
    rng = np.random.default_rng(2)
    gv = check_fd(verts, faces, ta, 1, rng.choice(len(verts), 6, replace=False))
    # translation invariance: the gradients of every result sum to zero over the vertices
    assert np.all(np.abs(gv.sum(axis=1)) <= 1e-9 * np.abs(gv).max(axis=(1, 2))[:, None])


def test_adjoint_two_surfaces_without_area_correction():
    tri, ta, tv = golden_mesh("1aki49_atom_01806")
    # shared vertices of the triangle soup (COMPON joins triangles on identical corners)
    verts, inv = np.unique(tri.reshape(-1, 3), axis=0, return_inverse=True)
    faces = inv.reshape(-1, 3)
    rng = np.random.default_rng(2)
    check_fd(verts, faces, None, 0, rng.choice(len(verts), 4, replace=False))


def test_gradient_needs_the_fp64_factors():
    verts, faces, ta, tv = meshes.ellipsoid_vf(4)
    st = bh.Setup(meshes.to_triangles(verts, faces), 1, ta)
    s = bh.BhmSolver()
    s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    xmu, gdef = st.deflation(s.diag_mean())
    bh.set_precision(bh.BGPU_MIXED)
    s.build(eps=1e-10, direct=0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
    bh.set_precision(-1)
    with pytest.raises(bh.BestGpuError):
        s.gradient(iarea=1, truearea=ta)
    s.destroy()


def test_adjoint_matches_the_cpu_reference_gradient():
    """Against the complex-step derivatives of the CPU oracle (oracle/gradref.py): both are exact up
    to rounding, so they agree far below the finite differences' accuracy."""
    from oracle import gradref
    verts, faces, ta, tv = meshes.ellipsoid_vf(6)
    tri = meshes.to_triangles(verts, faces)
    _, s, st = values_of(tri, ta, 1)
    vals, g = s.gradient(iarea=1, truearea=ta)
    bh.set_precision(-1)
    gv = meshes.corner_to_vertex(g, faces, len(verts))
    rng = np.random.default_rng(2)
    picks = [(int(v), int(c)) for v in rng.choice(len(verts), 4, replace=False) for c in range(3)]
    ref = gradref.gradient(verts, faces, 1, ta, picks)
    got = np.array([[gv[k, v, c] for (v, c) in picks] for k in range(3)])
    err = np.abs(got - ref).max(axis=1) / np.abs(gv).reshape(3, -1).max(axis=1)
    print(f"\nadjoint vs complex-step CPU reference: D_t {err[0]:.1e}, D_r {err[1]:.1e}, CHI' {err[2]:.1e}")
    assert np.all(err < 1e-9), err


def test_torch_autograd_wrapper():
    """The adjoint through torch.autograd (tests/torch_best.py): a scalar loss of the three results
    back-propagates to the vertices as the chain rule of the adjoint gradients says."""
    import torch
    from tests.torch_best import BestValues
    verts, faces, ta, tv = meshes.ellipsoid_vf(4)
    v = torch.tensor(verts, dtype=torch.float64, requires_grad=True)
    vals = BestValues.apply(v, faces, ta, 1)
    w = torch.tensor([1e6, 1e-7, 1e-4], dtype=torch.float64)
    (w * vals).sum().backward()
    _, s, st = values_of(meshes.to_triangles(verts, faces), ta, 1)
    _, g = s.gradient(iarea=1, truearea=ta)
    bh.set_precision(-1)
    gv = meshes.corner_to_vertex(g, faces, len(verts))
    expect = np.einsum("k,kvc->vc", w.numpy(), gv)
    assert np.allclose(v.grad.numpy(), expect, rtol=1e-12, atol=1e-12 * np.abs(expect).max())
