"""GPU tests of the mixed-precision path: the tcgen05 BF16 GEMM against an FP64 product of the
same BF16-rounded operands, and the refined solve (BF16 tensor-core LU + FP64 GMRES-IR) through
BEST's seam against the oracle.  Bars: GEMM within 1e-6 of k max|A| max|B| (FP32 accumulation);
D_t, D_r, D_tr, centres and CHI' within 1e-8 relative of the FP64 oracle (the metric's bar); golden
results at their 2e-4; a refinement that cannot converge falls back to the FP64 LU on the GPU."""
import numpy as np
import pytest

import best_hydro_b200 as bh
from oracle import best as ob
from best_hydro_b200 import BhmSolver, meshes
from tests.helpers import expected_cases, golden_mesh, rel, run_gpu, value_for_label

pytestmark = pytest.mark.gpu
TOL = 1e-8


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (300, 500, 70), (1000, 1000, 1000), (4096, 2048, 512),
                                   (129, 257, 65), (2000, 64, 4000)])
def test_tc_gemm_bf16(m, n, k):
    torch = _torch()
    g = torch.Generator().manual_seed(m + n + k)
    A = torch.randn(k, m, generator=g, dtype=torch.float32)  # column-major m x k: A.T
    B = torch.randn(n, k, generator=g, dtype=torch.float32)  # column-major k x n: B.T
    C = torch.randn(n, m, generator=g, dtype=torch.float32)  # column-major m x n: C.T
    dA, dB, dC = A.cuda(), B.cuda(), C.cuda()
    torch.cuda.synchronize()
    bh.gemm_bf16_minus_device(m, n, k, dA.data_ptr(), m, dB.data_ptr(), k, dC.data_ptr(), m)
    got = dC.cpu().double().T
    Ab = A.T.bfloat16().double()
    Bb = B.T.bfloat16().double()
    want = C.T.double() - Ab @ Bb
    err = (got - want).abs().max().item() / (Ab.abs().max().item() * Bb.abs().max().item() * k)
    assert err < 1e-6, err


@pytest.mark.parametrize("h", [128, 100, 42, 1])
def test_lu32_leaf(h):
    """The mixed LU's diagonal leaf: L U = A, L L^-1 = I and U U^-1 = I to FP32 accuracy (2e-5 of
    the scales, computed in FP64 from the FP32 results), the inverses zero outside h x h, and the
    padded block (ragged last leaf) handled."""
    torch = _torch()
    rng = np.random.default_rng(h)
    lda = 132
    A = np.zeros((lda, h), dtype=np.float32)  # column-major h x h with leading dimension lda: A[:h].T
    A[:h, :h] = (rng.standard_normal((h, h)) + 2.0 * np.sqrt(h) * np.eye(h)).astype(np.float32)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dL = torch.full((128, 128), 7.0, dtype=torch.float32, device="cuda")
    dU = torch.full((128, 128), 7.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    bh.lu32_leaf_device(h, dA.data_ptr(), lda, dL.data_ptr(), dU.data_ptr())
    out = dA.cpu().numpy().T[:h, :h].astype(np.float64)
    LI = dL.cpu().numpy().T.astype(np.float64)  # column-major 128 x 128
    UI = dU.cpu().numpy().T.astype(np.float64)
    L = np.tril(out, -1) + np.eye(h)
    U = np.triu(out)
    A64 = A[:h, :h].astype(np.float64)
    assert np.max(np.abs(L @ U - A64)) / np.max(np.abs(A64)) < 2e-5
    assert np.max(np.abs(L @ LI[:h, :h] - np.eye(h))) < 2e-5
    assert np.max(np.abs(U @ UI[:h, :h] - np.eye(h))) < 2e-5
    assert np.all(np.diag(LI[:h, :h]) == 1)
    assert np.all(np.triu(LI[:h, :h], 1) == 0) and np.all(np.tril(UI[:h, :h], -1) == 0)
    assert np.all(LI[h:, :] == 0) and np.all(LI[:, h:] == 0) and np.all(UI[h:, :] == 0) and np.all(UI[:, h:] == 0)


@pytest.mark.parametrize("left,kd,p0,length", [(True, 128, 256, 344), (False, 256, 32, 568), (True, 512, 0, 512),
                                               (False, 512, 96, 416), (True, 0, 128, 96)])
def test_trsm_leaf_tc(left, kd, p0, length):
    """The LU's triangular-solve leaf on the tensor cores (TF32 operands, FP32 accumulation): the
    block (h rows from kd x length columns from p0, or length rows x h columns) times the inverse
    diagonal block, against an FP64 product, within 2^-8 of |Dinv| |B| (TF32 rounding of both
    operands); the BF16 mirror equal to the result rounded to nearest; everything outside the block
    untouched.  n = 600: the last leaf is ragged (h = 88), as are the last tiles."""
    torch = _torch()
    n, lda, ldm = 600, 604, 640
    nleaves = (n + 127) // 128
    h = min(128, n - kd)
    rng = np.random.default_rng(kd * 7 + p0 + length + int(left))
    A = rng.standard_normal((n, n)).astype(np.float32)  # the matrix, A[i, j]
    D = np.zeros((nleaves, 128, 128), dtype=np.float32)  # D[b][i, k]: block b's inverse
    for b in range(nleaves):
        hb = min(128, n - 128 * b)
        D[b, :hb, :hb] = rng.standard_normal((hb, hb)).astype(np.float32) / np.sqrt(hb)
    dA = torch.zeros((n, lda), dtype=torch.float32)
    dA[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T))  # column j at row j
    dA = dA.cuda()
    # column-major 128 x 128 blocks, stacked: element (i, k) of block b at b*16384 + k*128 + i
    dD = torch.from_numpy(np.ascontiguousarray(np.transpose(D, (0, 2, 1)))).cuda()
    dZ = torch.full_like(dD, float("nan"))  # the unused inverse: never read
    mirror = torch.full((n, ldm), 3.0, dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    dl, du = (dD, dZ) if left else (dZ, dD)
    bh.trsm_leaf_device(left, n, dA.data_ptr(), lda, dl.data_ptr(), du.data_ptr(), kd, p0, h, length,
                        mirror.data_ptr(), ldm)
    got_all = dA.cpu().numpy()[:, :n].T.astype(np.float64)  # got_all[i, j]
    Dk = D[kd // 128, :h, :h].astype(np.float64)
    A64 = A.astype(np.float64)
    if left:
        blk = (slice(kd, kd + h), slice(p0, p0 + length))
        want = Dk @ A64[blk]
        bound = np.abs(Dk) @ np.abs(A64[blk])
    else:
        blk = (slice(p0, p0 + length), slice(kd, kd + h))
        want = A64[blk] @ Dk
        bound = np.abs(A64[blk]) @ np.abs(Dk)
    got = got_all[blk]
    assert np.all(np.abs(got - want) <= 2.0 ** -8 * bound + 1e-30), np.max(np.abs(got - want) / bound)
    outside = np.ones((n, n), dtype=bool)
    outside[blk] = False
    assert np.array_equal(got_all[outside], A64[outside])
    # the mirror: left column-major (element (i, j) at row j of the torch array), right row-major
    mir = mirror.float().cpu().numpy()
    mir_blk = mir[:, :n].T[blk] if left else mir[:, :n][blk]
    want_mir = torch.from_numpy(got.astype(np.float32)).bfloat16().float().numpy()
    assert np.array_equal(mir_blk, want_mir)
    mir_out = (mir[:, :n].T if left else mir[:, :n])[outside]
    assert np.all(mir_out == 3.0)


@pytest.mark.parametrize("left,kd,p0,length", [(True, 256, 512, 256), (False, 128, 384, 384), (True, 0, 256, 200),
                                               (False, 512, 0, 96), (True, 384, 640, 128)])
def test_trsm_leaf256_tc(left, kd, p0, length):
    """The LU's 256-deep triangular-solve leaf (k_combine256 + k_leaf256_tf32): the 256 x 256
    diagonal block's inverse formed from its two 128-block inverses, applied to the panel in place,
    against FP64 within 2^-8 of |T^-1| |P| (TF32 operands); the BF16 mirror equal to the result rounded
    to nearest; everything outside the panel untouched; whole and ragged tiles."""
    torch = _torch()
    n, lda, ldm = 768, 772, 768
    nleaves = n // 128
    rng = np.random.default_rng(kd + 3 * p0 + length + int(left))
    A = rng.standard_normal((n, n))
    for b in range(nleaves):  # well-conditioned diagonal blocks: small L, dominant U diagonal
        sl = slice(128 * b, 128 * b + 128)
        blk = A[sl, sl]
        A[sl, sl] = np.tril(blk, -1) * 0.3 / np.sqrt(128) + np.triu(blk, 1) * 0.3 / np.sqrt(128) + np.diag(
            2.0 + np.abs(np.diag(blk)))
    sl2 = slice(kd, kd + 256)
    A[kd + 128:kd + 256, kd:kd + 128] *= 0.3 / np.sqrt(128)  # L21
    A[kd:kd + 128, kd + 128:kd + 256] *= 0.3 / np.sqrt(128)  # U12
    A = A.astype(np.float32).astype(np.float64)
    DL = np.zeros((nleaves, 128, 128))
    DU = np.zeros((nleaves, 128, 128))
    for b in range(nleaves):
        blk = A[128 * b:128 * b + 128, 128 * b:128 * b + 128]
        DL[b] = np.linalg.inv(np.tril(blk, -1) + np.eye(128))
        DU[b] = np.linalg.inv(np.triu(blk))
    dA = torch.zeros((n, lda), dtype=torch.float32)
    dA[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T).astype(np.float32))
    dA = dA.cuda()
    dDL = torch.from_numpy(np.ascontiguousarray(np.transpose(DL, (0, 2, 1))).astype(np.float32)).cuda()
    dDU = torch.from_numpy(np.ascontiguousarray(np.transpose(DU, (0, 2, 1))).astype(np.float32)).cuda()
    mirror = torch.full((n, ldm), 3.0, dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    bh.trsm_leaf256_device(left, n, dA.data_ptr(), lda, dDL.data_ptr(), dDU.data_ptr(), kd, p0, length,
                           mirror.data_ptr(), ldm)
    got_all = dA.cpu().numpy()[:, :n].T.astype(np.float64)
    T = A[sl2, sl2]
    if left:
        Tinv = np.linalg.inv(np.tril(T, -1) + np.eye(256))
        blk = (sl2, slice(p0, p0 + length))
        want, bound = Tinv @ A[blk], np.abs(Tinv) @ np.abs(A[blk])
    else:
        Tinv = np.linalg.inv(np.triu(T))
        blk = (slice(p0, p0 + length), sl2)
        want, bound = A[blk] @ Tinv, np.abs(A[blk]) @ np.abs(Tinv)
    got = got_all[blk]
    assert np.all(np.abs(got - want) <= 2.0 ** -8 * bound + 1e-30), np.max(np.abs(got - want) / bound)
    outside = np.ones((n, n), dtype=bool)
    outside[blk] = False
    assert np.array_equal(got_all[outside], A[outside])
    mir = mirror.float().cpu().numpy()
    mir_blk = mir[:, :n].T[blk] if left else mir[:, :n][blk]
    want_mir = torch.from_numpy(got.astype(np.float32)).bfloat16().float().numpy()
    assert np.array_equal(mir_blk, want_mir)
    assert np.all((mir[:, :n].T if left else mir[:, :n])[outside] == 3.0)


@pytest.mark.parametrize("m,nc", [(128, 300), (300, 100), (50, 384), (128, 128), (384, 7), (256, 384), (384, 200)])
def test_panel_update_tc(m, nc):
    """The LU's K = 128 update on the tensor cores (TF32 operands, FP32 accumulation): C -= A B with
    one side at most 256 (the left form for m <= nc, the right one otherwise), against FP64 within
    2^-8 of |A| |B|; everything outside C untouched; ragged sizes; a short side of 129-256 in two
    row groups."""
    torch = _torch()
    n, lda = 640, 644
    ar, ac, br, bc, cr, cc = 0, 0, 128, 128, 256, 256
    rng = np.random.default_rng(m * 1000 + nc)
    A = rng.standard_normal((n, n)).astype(np.float32)
    dA = torch.zeros((n, lda), dtype=torch.float32)
    dA[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T))
    dA = dA.cuda()
    torch.cuda.synchronize()
    bh.panel_update_device(n, dA.data_ptr(), lda, m, nc, ar, ac, br, bc, cr, cc)
    got_all = dA.cpu().numpy()[:, :n].T.astype(np.float64)
    A64 = A.astype(np.float64)
    a, b = A64[ar:ar + m, ac:ac + 128], A64[br:br + 128, bc:bc + nc]
    blk = (slice(cr, cr + m), slice(cc, cc + nc))
    want = A64[blk] - a @ b
    bound = np.abs(a) @ np.abs(b)
    err = np.abs(got_all[blk] - want)
    assert np.all(err <= 2.0 ** -8 * bound + 1e-6 * np.abs(A64[blk])), np.max(err / bound)
    outside = np.ones((n, n), dtype=bool)
    outside[blk] = False
    assert np.array_equal(got_all[outside], A64[outside])


def compare(g, o, tol=TOL):
    for key in ("Dtt", "Drr"):
        assert rel(g["tensors"][key], o.tensors[key]) < tol, key
    scale = np.sqrt(np.max(np.abs(o.tensors["Dtt"])) * np.max(np.abs(o.tensors["Drr"])))
    assert np.max(np.abs(g["tensors"]["Dtr"] - o.tensors["Dtr"])) / scale < tol
    size = np.sqrt(np.mean(o.x.reshape(3, -1) ** 2) * 3)
    for key in ("urc", "udr"):
        assert np.max(np.abs(g["tensors"][key] - o.tensors[key])) / size < tol
    if o.chiprime is not None:
        assert abs(g["chiprime"] / o.chiprime - 1) < tol


@pytest.mark.parametrize("case", ["icosphere_1280", "ellipsoid_5120", "star_f16"])
def test_mixed_solve_vs_oracle(case):
    if case == "icosphere_1280":
        (tri, ta, tv), iarea = meshes.icosphere(3, 20.0), 1
    elif case == "ellipsoid_5120":
        (tri, ta, tv), iarea = meshes.ellipsoid(16), 1
    else:
        (tri, ta, tv), iarea = meshes.star(16), 0
    bh.set_precision(bh.BGPU_MIXED)
    try:
        solver = BhmSolver()
        g = run_gpu(solver, tri, ta, iarea=iarea, direct=0, eps=1e-10, ivisco=1, truevol=tv)
        logs = bh.log_lines()
        t = bh.timings()
        solver.destroy()
    finally:
        bh.set_precision(-1)
    print(f"\n{case}: {t} | {' / '.join(l for l in logs if 'solve' in l or 'build' in l)}")
    assert not any("instead" in l for l in logs), logs
    # a few GMRES iterations (3-5 at these sizes): a factor gone wrong would still converge, slowly
    assert 0 < t["refine_iters"] <= 12 and t["relres"] <= 1e-12, t
    o = ob.best_run(tri, ta, tv, iarea=iarea, ivisco=1)
    compare(g, o)


def test_mixed_operand_copies_in_blocks(monkeypatch):
    """The path without BF16 mirrors (when the GPU has no room for them): operands copied per
    product into buffers of capped rows, so the large products run in blocks."""
    monkeypatch.setenv("BEST_GPU_NO_MIRRORS", "1")
    monkeypatch.setenv("BEST_GPU_OPERAND_ROWS", "1024")
    tri, ta, tv = meshes.ellipsoid(12)
    bh.set_precision(bh.BGPU_MIXED)
    try:
        solver = BhmSolver()
        g = run_gpu(solver, tri, ta, iarea=1, direct=0, eps=1e-10, ivisco=1, truevol=tv)
        logs = bh.log_lines()
        t = bh.timings()
        solver.destroy()
    finally:
        bh.set_precision(-1)
    assert not any("instead" in l for l in logs), logs
    # a few GMRES iterations (3-5 at these sizes): a factor gone wrong would still converge, slowly
    assert 0 < t["refine_iters"] <= 12 and t["relres"] <= 1e-12, t
    compare(g, ob.best_run(tri, ta, tv, iarea=1, ivisco=1))


def test_mixed_golden_2eu7():
    c = expected_cases()["2eu7"]
    tri, ta, tv = golden_mesh(c["mesh"])
    bh.set_precision(bh.BGPU_MIXED)
    try:
        solver = BhmSolver()
        g = run_gpu(solver, tri, ta, iarea=1, direct=0, eps=1e-10, ivisco=1, truevol=tv, wm=c["wm"])
        solver.destroy()
    finally:
        bh.set_precision(-1)
    for e in c["expected"]:
        got = value_for_label(g["report"], e["label"])
        assert abs(got - e["value"]) <= e["tol"] * abs(e["value"]), (e["label"], got)
    compare(g, ob.best_run(tri, ta, tv, iarea=1, ivisco=1, wm=c["wm"]))


def test_mixed_falls_back_to_fp64_when_refinement_cannot_converge():
    """No restarts allowed: the refinement cannot reach its tolerance, so bhm_solve factors the kept
    FP64 matrix on the GPU and returns the FP64 solution (a host-side failure, no GPU fault)."""
    tri, ta, tv = meshes.icosphere(2, 20.0)
    bh.set_precision(bh.BGPU_MIXED)
    bh.set_refinement(0, 10)
    try:
        solver = BhmSolver()
        g = run_gpu(solver, tri, ta, iarea=1, direct=0, eps=1e-10)
        logs = bh.log_lines()
        solver.destroy()
    finally:
        bh.set_precision(-1)
        bh.set_refinement(8, 10)
    assert any("factoring the FP64 matrix instead" in l for l in logs), logs
    compare(g, ob.best_run(tri, ta, tv, iarea=1), tol=1e-10)
