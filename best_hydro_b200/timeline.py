"""Per-launch durations of the mixed LU's factorisation, from the launch stamps the library writes
when ``BEST_GPU_TIMELINE=<file>`` is set (one ``slot,kind,flops,start_ns,end_ns`` line per stamped
launch, appended per factorisation; kinds 0 BF16 GEMM, 1 LU leaf or 256-block inverses, 2
triangular-solve leaf, 3 small FP32 update, 4 TF32 panel update).

    python -m best_hydro_b200.timeline DUMP.csv N3

labels each launch of the last factorisation in the file with its shape by replaying the LU's
recursion (``MixedSolver::rlu`` / ``trsm_llu`` / ``trsm_ru`` / ``gemm`` in csrc/mixed.cu, in launch
order) and prints, per shape class, the count and the sum, median, minimum and maximum of the
launches' first-CTA-start to last-CTA-end times.  The two triangular-solve chains of a recursion
step run on two streams, so sums of concurrent classes exceed the wall time.
"""
import collections
import sys

import numpy as np

LEAF = 128


def _split(sz):
    return max((sz // 2) // LEAF * LEAF, LEAF)


def _update_kind(m, n, k):
    return "panel" if k == 128 and (min(m, n) <= 128 or (min(m, n) <= 256 and max(m, n) <= 3840)) else "gemm"


def launch_labels(n3):
    """(kind, m, n, k) of every stamped launch of the factorisation at order n3, in launch order:
    kind "lu" (diagonal leaf), "inv256" (a 256-block's inverses), "leafL" / "leafR" (triangular-solve
    leaves: h x w, m x h; k = their depth, 128 or 256), "panel" (TF32 panel update), "gemm" (BF16
    tensor-core GEMM)."""
    out = []

    def gemm(m, n, k):
        if m > 0 and n > 0 and k > 0:
            out.append((_update_kind(m, n, k), m, n, k))

    def trsm_left(h, w):
        if h <= 0 or w <= 0:
            return
        if h <= LEAF or h == 2 * LEAF:
            out.append(("leafL", h, w, h))
            return
        h1 = _split(h)
        trsm_left(h1, w)
        gemm(h - h1, w, h1)
        trsm_left(h - h1, w)

    def trsm_right(h, m):
        if h <= 0 or m <= 0:
            return
        if h <= LEAF or h == 2 * LEAF:
            out.append(("leafR", m, h, h))
            return
        h1 = _split(h)
        trsm_right(h1, m)
        gemm(m, h - h1, h1)
        trsm_right(h - h1, m)

    def rlu(sz):
        if sz <= LEAF:
            out.append(("lu", sz, sz, sz))
            return
        h = _split(sz)
        r = sz - h
        rlu(h)
        trsm_left(h, r)
        trsm_right(h, r)
        gemm(r, r, h)
        rlu(r)
        if sz == 2 * LEAF:
            out.append(("inv256", sz, sz, sz))

    rlu(n3)
    return out


def _class(kind, m, n, k):
    if kind in ("leafL", "leafR"):
        w = n if kind == "leafL" else m
        return f"{kind}{k} {'w<=256' if w <= 256 else ('w<=2048' if w <= 2048 else 'w>2048')}"
    if kind == "gemm" and max(m, n) >= 4096:
        return f"gemm large, k={k}"
    if kind in ("gemm", "panel", "small"):
        return f"{kind} {m}x{n}x{k}"
    return kind


def summarise(path, n3):
    rows = [line.strip().split(",") for line in open(path) if line.strip()]
    starts = [i for i, r in enumerate(rows) if r[0] == "0"]
    last = rows[starts[-1]:]
    labels = launch_labels(n3)
    if len(last) != len(labels):
        raise SystemExit(f"{len(last)} stamped launches in the last factorisation, {len(labels)} in the replay")
    t = np.array([[int(r[3]), int(r[4])] for r in last], dtype=np.int64)
    dur = (t[:, 1] - t[:, 0]) / 1e3
    lines = [f"span {(t[:, 1].max() - t[:, 0].min()) / 1e6:.1f} ms, {len(last)} stamped launches"]
    by = collections.defaultdict(list)
    for lab, d in zip(labels, dur):
        by[_class(*lab)].append(d)
    for key, ds in sorted(by.items(), key=lambda kv: -sum(kv[1])):
        ds = np.array(ds)
        lines.append(f"{key:<30} n={len(ds):5d}  sum {ds.sum() / 1e3:8.2f} ms  median {np.median(ds):8.1f} us  "
                     f"min {ds.min():8.1f}  max {ds.max():8.1f}")
    return lines


if __name__ == "__main__":
    print("\n".join(summarise(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 61440)))
