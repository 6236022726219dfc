"""CPU tests of the H-matrix path's host logic: the cluster tree and block partition of
bgpu_hmatrix_plan against the reference's algorithm restated in oracle/hplan.py
(hmatrix/src/cluster.cpp, hmatrix/src/hmatrix.cpp:26-53).  No GPU is used."""
import numpy as np
import pytest

import best_hydro_b200 as bh
from best_hydro_b200 import meshes
from oracle import best as ob
from oracle import hplan


def _mesh(kind):
    if kind == "ellipsoid":
        tri, ta, tv = meshes.ellipsoid(8)
    elif kind == "star32":
        tri, ta, tv = meshes.star(32)  # the benchmark's mesh, N = 20,480
    else:
        tri, ta, tv = meshes.star(10)
    s = ob.setup(tri, 1, ta)
    x, _ = ob.incenters_and_self(s)
    return s, x


@pytest.mark.parametrize("kind,leaf", [("ellipsoid", 32), ("ellipsoid", 128), ("star", 64), ("star32", 128)])
def test_plan_matches_reference_tree(kind, leaf):
    s, x = _mesh(kind)
    n = s.n
    v1, v2, v3 = s.colmajor()
    perm, counts = bh.hmatrix_plan(x, v1, v2, v3, leaf=leaf, eta=2.0, kmax=90)
    X = x.reshape(3, n).T
    corners = np.stack([s.v1, s.v2, s.v3], 1)
    cl, depth, _ = hplan.cluster_tree(X, corners, leaf)
    assert counts["depth"] == depth
    assert sorted(perm.tolist()) == list(range(n))
    leaves = [c for c in cl if c["sons"] is None]
    assert counts["leaves"] == len(leaves)
    # every leaf of the reference tree is a contiguous range of the library's tree order, in order
    pos = 0
    for c in sorted(leaves, key=lambda c: c["beg"]):
        assert frozenset(perm[pos:pos + c["cnt"]].tolist()) == c["members"]
        pos += c["cnt"]
    blk = hplan.blocks(cl, 2.0)
    adm = [b for b in blk if b[2]]
    assert counts["admissible"] == len(adm)
    assert counts["dense"] + counts["lowrank"] == len(blk)
    # an admissible block is low-rank exactly when 9 nr nc > 3 (nr + nc) kmax
    low = sum(1 for t, s_, a in blk if a and 9 * cl[t]["cnt"] * cl[s_]["cnt"] > 3 * (cl[t]["cnt"] + cl[s_]["cnt"]) * 90)
    assert counts["lowrank"] == low


def test_plan_covers_every_pair_once():
    s, x = _mesh("ellipsoid")
    n = s.n
    X = x.reshape(3, n).T
    corners = np.stack([s.v1, s.v2, s.v3], 1)
    cl, _, _ = hplan.cluster_tree(X, corners, 32)
    cover = np.zeros((n, n), dtype=np.int32)
    for t, s_, _ in hplan.blocks(cl, 2.0):
        rows = np.array(sorted(cl[t]["members"]))
        cols = np.array(sorted(cl[s_]["members"]))
        cover[np.ix_(rows, cols)] += 1
    assert (cover == 1).all()


def test_plan_rejects_bad_options():
    s, x = _mesh("ellipsoid")
    with pytest.raises(bh.BestGpuError):
        bh.hmatrix_set_options(leaf=4)
    with pytest.raises(bh.BestGpuError):
        bh.hmatrix_set_options(kmax=91)
    bh.hmatrix_set_options()
