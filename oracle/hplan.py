"""Test infrastructure (the oracle): the reference H-matrix's cluster tree and block partition,
restated in numpy for checking the library's plan (bgpu_hmatrix_plan).  Not part of the product.

hmatrix/src/cluster.cpp:93-113 (build_cluster_tree: the depth, the root), :10-74 (split: corner box,
incenter extent, median split by (coordinate, index)), :76-91 (diam, dist), :115-117 (admissible);
hmatrix/src/hmatrix.cpp:26-53 (make_blocks: admissible -> low-rank candidate, a leaf pair -> dense,
else the four son pairs).
"""
import numpy as np


def cluster_tree(x, corners, leaf):
    """x: (n, 3) incenters, corners: (n, 3, 3).  Returns (clusters, leaves): clusters as dicts with
    beg, cnt, lo, hi, sons (None for a leaf) and the member triangles (a set per cluster)."""
    n = x.shape[0]
    depth = 0
    while (n + (1 << depth) - 1) >> depth > leaf:
        depth += 1
    perm = np.arange(n)
    cl = []

    def split(beg, cnt, lev):
        idx = perm[beg:beg + cnt].copy()
        pts = corners[idx].reshape(-1, 3)
        cid = len(cl)
        cl.append(dict(beg=beg, cnt=cnt, lo=pts.min(0), hi=pts.max(0), sons=None, level=lev))
        if lev == depth:
            return cid
        xi = x[idx]
        ext = xi.max(0) - xi.min(0)
        axis = 0
        for d in (1, 2):
            if ext[d] > ext[axis]:
                axis = d
        order = np.lexsort((idx, xi[:, axis]))  # by coordinate, ties by triangle index
        perm[beg:beg + cnt] = idx[order]
        h = cnt // 2
        a = split(beg, h, lev + 1)
        b = split(beg + h, cnt - h, lev + 1)
        cl[cid]["sons"] = (a, b)
        return cid

    split(0, n, 0)
    for c in cl:
        c["members"] = frozenset(perm[c["beg"]:c["beg"] + c["cnt"]].tolist())
    return cl, depth, perm


def blocks(cl, eta):
    """(t, s, admissible) for every leaf of the block tree."""
    def diam(c):
        return float(np.sqrt(np.sum((cl[c]["hi"] - cl[c]["lo"]) ** 2)))

    def dist(a, b):
        gap = np.maximum(0.0, np.maximum(cl[a]["lo"] - cl[b]["hi"], cl[b]["lo"] - cl[a]["hi"]))
        return float(np.sqrt(np.sum(gap * gap)))

    out = []
    stack = [(0, 0)]
    while stack:
        t, s = stack.pop()
        if t != s and min(diam(t), diam(s)) <= eta * dist(t, s):
            out.append((t, s, True))
        elif cl[t]["sons"] is None or cl[s]["sons"] is None:
            out.append((t, s, False))
        else:
            for p in cl[t]["sons"]:
                for q in cl[s]["sons"]:
                    stack.append((p, q))
    return out
