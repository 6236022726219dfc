"""What BEST's GR check (BEST_HMATRIX_CHECK, best/besolve.f90:245-277) counts with the GPU backend.

The GPU's exact entries are TGETGR's arithmetic (best/tgetgr.f, best/triangleint.f) with correctly
rounded acos/sin/cos/log; the reference calls glibc's, which are not correctly rounded everywhere
(glibc's log is off by one ulp on about 0.15 % of arguments).  These CPU tests account for every
entry where the two differ, on the reference's example meshes:
  * the differing entries are exactly the committed list (tests/golden/hmcheck_glibc_misrounds.npz,
    made by tests/golden/make_hmcheck_list.py);
  * each lies in a triangle pair whose GR block calls glibc at an argument where glibc's result is
    not the correctly rounded one (the correctly rounded functions are checked against exact
    decimal arithmetic in tests/test_ddmath.py);
  * incenters, which involve no transcendental function, agree bit for bit.
The GPU test tests/test_gpu_assembly.py::test_hmcheck_2eu7 shows the GPU's entries equal the
correctly rounded evaluation everywhere, so the GR check reports exactly these entries.
"""
import numpy as np
import pytest

from oracle import best as ob
from tests import crshim
from tests.golden.make_hmcheck_list import MESHES, differing_entries
from tests.helpers import GOLDEN, golden_mesh


@pytest.mark.parametrize("name", MESHES)
def test_differences_from_reference_are_glibc_misrounds(name):
    d, s = differing_entries(name)
    g = np.load(f"{GOLDEN}/hmcheck_glibc_misrounds.npz")
    assert int(g[name + "_order"]) == 3 * s.n
    assert np.array_equal(d, g[name])
    # about 0.06 % of the entries
    assert 0 < len(d) < 1e-3 * (3 * s.n) ** 2
    pairs = np.unique(d // 3, axis=0)
    x, _ = ob.incenters_and_self(s, 1.0)
    cnt = crshim.fn_misrounds(s, x, pairs[:, 0], pairs[:, 1])
    assert np.all(cnt > 0), pairs[cnt == 0][:10]
    xc, _ = crshim.self_blocks_cr(s, 1.0)
    assert np.array_equal(x.view(np.int64), xc.view(np.int64))


def test_pairs_without_misrounds_are_identical():
    """The converse on a sample: pairs whose calls glibc all rounds correctly have identical blocks."""
    name = "1aki49_atom_01806"
    tri, ta, tv = golden_mesh(name)
    s = ob.setup(tri, 1, ta)
    rng = np.random.default_rng(7)
    n1 = rng.integers(0, s.n, 400)
    n2 = rng.integers(0, s.n, 400)
    x, self9 = ob.incenters_and_self(s, 1.0)
    cnt = crshim.fn_misrounds(s, x, n1, n2)
    ref, _, _ = ob.assemble(s, 1.0)
    cr, _, _ = crshim.assemble_cr(s, 1.0)
    for a, b, c in zip(n1, n2, cnt):
        if c == 0:
            blk_r = ref[3 * a:3 * a + 3, 3 * b:3 * b + 3]
            blk_c = cr[3 * a:3 * a + 3, 3 * b:3 * b + 3]
            assert np.array_equal(blk_r.view(np.int64), blk_c.view(np.int64)), (a, b)
