"""Single-kernel cases for profiling (one warm-up launch, then the launch to capture).

    python -m best_hydro_b200.kernel_cases tc_gemm M N K     # C -= A B, BF16 tcgen05 (FP32 C)
    python -m best_hydro_b200.kernel_cases dgemm M N K       # C -= A B, FP64 DMMA
    python -m best_hydro_b200.kernel_cases assemble F [mixed]  # GR of the ellipsoid at geodesic frequency F
                                                             # (mixed: the mixed path's assembly)
    python -m best_hydro_b200.kernel_cases mixed F           # mixed build + solve, ellipsoid frequency F
    python -m best_hydro_b200.kernel_cases adjoint F         # FP64 build + adjoint gradients (k_pair_adjoint)
    python -m best_hydro_b200.kernel_cases hmatrix F [EPS]  # H-matrix build + 6-RHS GMRES solve of the star
                                                             # body at geodesic frequency F (eps 1e-4), then
                                                             # five timed 6-column products
    python -m best_hydro_b200.kernel_cases panel left|right leaf|update LEN
                                                             # k_panel_tf32: a triangular-solve leaf or a
                                                             # K = 128 update on a 128 x LEN panel

Each case launches its kernel twice (the second launch is the one to capture: `ncu -k <kernel>
-s 1 -c 1`) and prints the CUDA-event time of the second launch.
"""
import sys


def _ev(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def main(argv):
    import torch

    import best_hydro_b200 as bh
    case = argv[0]
    dev = torch.device("cuda", 0)
    if case in ("tc_gemm", "dgemm"):
        m, n, k = (int(v) for v in argv[1:4])
        dt = torch.float32 if case == "tc_gemm" else torch.float64
        g = torch.Generator(device=dev).manual_seed(0)
        a = torch.randn(k, m, dtype=dt, device=dev, generator=g)  # a[j] = column j: column-major m x k
        b = torch.randn(n, k, dtype=dt, device=dev, generator=g)
        c = torch.randn(n, m, dtype=dt, device=dev, generator=g)
        fn = bh.gemm_bf16_minus_device if case == "tc_gemm" else bh.dgemm_minus_device
        kid = bh.BGPU_KERNEL_TC_GEMM if case == "tc_gemm" else bh.BGPU_KERNEL_LU_GEMM64
        reps = int(argv[4]) if len(argv) > 4 else 1
        fn(m, n, k, a.data_ptr(), m, b.data_ptr(), k, c.data_ptr(), m)
        torch.cuda.synchronize()
        bh.kernel_stats(kid, enable=1)
        e0, e1 = _ev(torch)
        e0.record()
        for _ in range(reps):
            fn(m, n, k, a.data_ptr(), m, b.data_ptr(), k, c.data_ptr(), m)
        e1.record()
        torch.cuda.synchronize()
        launches, kms, work = bh.kernel_stats(kid, enable=0)
        call = e0.elapsed_time(e1) / reps
        if launches:
            kms /= launches
            print(f"{case} {m}x{n}x{k}: kernel {kms:.3f} ms, {2.0 * m * n * k / kms / 1e9:.1f} TFLOP/s "
                  f"(whole call {call:.3f} ms)")
        else:
            print(f"{case} {m}x{n}x{k}: call {call:.3f} ms, {2.0 * m * n * k / call / 1e9:.1f} TFLOP/s")
        return 0
    if case == "panel":
        left, leaf, length = argv[1] == "left", argv[2] == "leaf", int(argv[3])
        n = length + 256
        lda = (n + 3) // 4 * 4
        g = torch.Generator(device=dev).manual_seed(0)
        a = torch.randn(n, lda, dtype=torch.float32, device=dev, generator=g)  # a[j] = column j
        nleaves = (n + 127) // 128
        d = torch.randn(nleaves, 128, 128, dtype=torch.float32, device=dev, generator=g) / 16
        mir = torch.zeros(n, lda, dtype=torch.bfloat16, device=dev)
        torch.cuda.synchronize()
        for _ in range(2):
            if leaf:
                # left: rows [0, 128) x columns [256, 256 + LEN); right: rows [256, ..) x columns [0, 128)
                bh.trsm_leaf_device(left, n, a.data_ptr(), lda, d.data_ptr(), d.data_ptr(), 0, 256, 128, length,
                                    mir.data_ptr(), lda)
            elif left:
                bh.panel_update_device(n, a.data_ptr(), lda, 128, length, 128, 0, 0, 256, 128, 256)
            else:
                bh.panel_update_device(n, a.data_ptr(), lda, length, 128, 256, 0, 0, 128, 256, 128)
        torch.cuda.synchronize()
        print(f"panel {'left' if left else 'right'} {'leaf' if leaf else 'update'} 128 x {length}: done")
        return 0
    if case == "adjoint":
        from best_hydro_b200 import meshes
        f = int(argv[1])
        tri, ta, tv = meshes.ellipsoid(f)
        st = bh.Setup(tri, 1, ta)
        s = bh.BhmSolver()
        s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        xmu, gdef = st.deflation(s.diag_mean())
        bh.set_precision(bh.BGPU_FP64)
        s.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        for _ in range(2):
            s.gradient(iarea=1, truearea=ta)
        print([ln for ln in bh.log_lines() if ln.startswith("gradient")][-1])
        return 0
    if case == "hmatrix":
        from best_hydro_b200 import meshes
        f = int(argv[1])
        eps = float(argv[2]) if len(argv) > 2 else 1e-4
        tri, ta, tv = meshes.star(f)
        st = bh.Setup(tri, 0, ta)
        s = bh.BhmSolver()
        s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        x = s.incenters()
        xmu, gdef = st.deflation(s.diag_mean())
        bh.set_precision(bh.BGPU_HMATRIX)
        s.build(eps=eps, direct=0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        s.solve(bh.rhs6(x))
        t = bh.timings()
        hs = bh.hmatrix_stats()
        n3 = 3 * st.n
        xs = torch.randn(6, n3, dtype=torch.float64, device=dev)
        ys = torch.empty_like(xs)
        ls = torch.cuda.ExternalStream(bh.lib().bgpu_stream())  # the library's stream, where it launches
        e0, e1 = _ev(torch)
        torch.cuda.synchronize()
        e0.record(ls)
        for _ in range(5):
            bh.hmatrix_matvec_device(6, xs.data_ptr(), n3, ys.data_ptr(), n3)
        e1.record(ls)
        torch.cuda.synchronize()
        mv = e0.elapsed_time(e1) / 5
        gb = 8 * (hs["dense_entries"] + hs["lowrank_entries"]) / 1e9
        print(f"hmatrix N={st.n} eps={eps:g}: build {t['build']:.1f} ms (fill {hs['fill_ms']:.1f}, ACA "
              f"{hs['aca_ms']:.1f}, preconditioner {hs['precond_ms']:.1f}), solve {t['solve']:.1f} ms "
              f"({int(hs['gmres_steps'])} GMRES steps); product of 6 columns {mv:.3f} ms over {gb:.2f} GB "
              f"({gb / mv * 1e3:.0f} GB/s of stored blocks)")
        for line in bh.log_lines():
            print(line)
        bh.set_precision(-1)
        return 0
    if case in ("assemble", "mixed"):
        f = int(argv[1])
        from best_hydro_b200 import meshes
        tri, ta, tv = meshes.ellipsoid(f)
        st = bh.Setup(tri, 1, ta)
        s = bh.BhmSolver()
        s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        n3 = 3 * st.n
        if case == "assemble":
            out = torch.empty((n3, n3), dtype=torch.float64, device=dev)
            for _ in range(2):
                e0, e1 = _ev(torch)
                torch.cuda.synchronize()
                e0.record()
                bh.assemble_device(0, st.n, 0, st.n, out.data_ptr(), n3, mixed=len(argv) > 2 and argv[2] == "mixed")
                e1.record()
                torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            kind = "mixed" if len(argv) > 2 and argv[2] == "mixed" else "exact"
            print(f"assemble ({kind}) N={st.n}: {ms:.3f} ms, {st.n * (st.n - 1) / ms / 1e6:.3f} Gpairs/s")
            return 0
        x = s.incenters()
        xmu, gdef = st.deflation(s.diag_mean())
        bh.set_precision(bh.BGPU_MIXED)
        for _ in range(2):
            s.build(eps=1e-10, direct=0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
            s.solve(bh.rhs6(x))
        t = bh.timings()
        print(f"mixed N={st.n}: factor {t['factor']:.2f} ms, solve {t['solve']:.2f} ms, "
              f"{int(t['refine_iters'])} iterations, residual {t['relres']:.2e}")
        for line in bh.log_lines():
            print(line)
        return 0
    print(__doc__)
    return 2


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
