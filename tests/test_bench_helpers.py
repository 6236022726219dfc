"""CPU checks of bench.py's accounting: the replay of the mixed LU's GEMM shapes gives the launch
count the library stamps (2,017 at order 61,440: 1,569 BF16 tensor-core GEMMs and 448 TF32 panel
updates; a triangular solve 256 deep is one leaf) and the LU's flop count, and the traffic estimate stays within the
measured per-class ratios."""
import bench


def test_lu_gemm_shapes_replay():
    shapes = bench.lu_gemm_shapes(61440)
    assert len(shapes) == 2017
    flops = sum(2 * m * n * k for m, n, k in shapes)
    n = 61440
    # (2/3) n^3 minus the diagonal leaves' and triangular-solve leaves' share
    assert 0.99 * (2 / 3) * n ** 3 < flops < (2 / 3) * n ** 3
    assert bench.lu_gemm_shapes(128) == []


def test_gemm_traffic_estimate_in_range():
    tr, alg, count = bench.gemm_traffic_per_launch(61440)
    lo, hi = min(bench.GEMM_TRAFFIC_RATIO.values()), max(bench.GEMM_TRAFFIC_RATIO.values())
    shapes = bench.lu_gemm_shapes(61440)
    panel = sum(1 for sh in shapes if bench.panel_update(*sh))
    assert panel == 448
    assert count == 2017 - panel == 1569 and lo * alg <= tr <= hi * alg
