#!/usr/bin/env python
"""Benchmark of BEST's dense hot path on the B200: seconds per BEST solve (assemble GR with the
deflation, LU, solve for the 6 translation/rotation right-hand sides).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload star_f32|ellipsoid_f16|icosphere_l3] [--precision mixed|fp64]

One JSON line on rank 0.  `value` is the device time per solve of the timed path (default: the
mixed-precision factorisation + FP64 GMRES refinement) with the mesh already in HBM (CUDA events on
the library's stream, L2 flushed between steps); `fp64_path` is the plain FP64 path timed the same
way, and `accuracy` the relative differences of D_t, D_r and [eta] (11-RHS solves) between the two.
`e2e` is the timed path through the C ABI with host buffers (bhm_create ... bhm_solve, copies
included).  With N GPUs (torchrun), every rank
solves its own replica: the path has no exchange step, so there is no collective in it.
`--impl reference` times the reference's own CPU implementation (its kernel.cpp assembly, OpenMP,
the deflation, and the LAPACK dgetrf/dgetrs BEST calls) on complete solves of the same workload: as
many as fit in --ref-budget-s seconds, at least one; `steps` is the number run.  The GPU arm's
`cpu_baseline` is one such complete solve, whose tensors are the oracle of `accuracy`.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s per BEST solve (assemble+LU+6 RHS), mixed vs FP64 GPU at rel err<=1e-8"

WORKLOADS = {
    # the headline workload: star body at geodesic frequency 32 (N = 20,480)
    "star_f32": dict(desc="star-shaped body r=25A(1+sum_{l=2..8} a_lm Y_lm), a_lm~N(0,(0.08/l)^2) seed 1, "
                          "geodesic f=32", N=20480, iarea=0, gen=("star", 32)),
    "star_f45": dict(desc="star-shaped body as star_f32, geodesic f=45 (the FP32 factor fits beside the FP64 GR)",
                     N=40500, iarea=0, gen=("star", 45)),
    "ellipsoid_f16": dict(desc="ellipsoid 30/20/12 A, geodesic f=16, normal jitter U(+-2%) seed 0", N=5120,
                          iarea=1, gen=("ellipsoid", 16)),
    "icosphere_l3": dict(desc="icosphere level 3, R=20 A", N=1280, iarea=1, gen=("icosphere", 3)),
    # the batching workload: the ellipsoid at eight geodesic frequencies, solved as one series
    # the differentiation workload: gradients of the ellipsoid at frequency 16 (N = 5,120)
    "ellipsoid_adjoint": dict(desc="ellipsoid 30/20/12 A, geodesic f=16, normal jitter U(+-2%) seed 0: adjoint "
                                   "gradients w.r.t. all 3 x 2562 vertex coordinates", N=5120, iarea=1,
                              gen=("adjoint", 16)),
    "ellipsoid_series": dict(desc="ellipsoid 30/20/12 A, normal jitter U(+-2%) seed 0, geodesic f = 11, 12, 14, "
                                  "16, 18, 20, 22, 23 (one series, FP64)", N=49080, iarea=1,
                             gen=("series", (11, 12, 14, 16, 18, 20, 22, 23))),
}


def make_mesh(name):
    from best_hydro_b200 import meshes
    kind, arg = WORKLOADS[name]["gen"]
    if kind == "series":
        return [meshes.ellipsoid(f) for f in arg]
    if kind == "adjoint":
        return meshes.ellipsoid(arg)
    if kind == "star":
        return meshes.star(arg)
    if kind == "ellipsoid":
        return meshes.ellipsoid(arg)
    return meshes.icosphere(arg, 20.0)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------------
# CPU baseline: the reference's own implementation on the host cores, on bounded samples
# ------------------------------------------------------------------------------------------------

def cpu_reference_sample(tri, iarea, truearea, rows=512, n_lu=12288, seed=0):
    """One bounded sample, scaled to a full solve: (seconds per solve, parts dict)."""
    import ctypes

    from oracle import best as ob
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    s = ob.setup(tri, iarea, truearea)
    n = s.n
    R = ob.ref_lib()
    kind = "reference"
    if R is None:
        kind = "port"
    v1, v2, v3 = s.colmajor()
    rows = min(rows, n)
    buf = np.empty((3 * rows, 3 * n), order="F")
    dp = ctypes.POINTER(ctypes.c_double)
    if R is not None:
        R.ref_create(n, v1.ctypes.data_as(dp), v2.ctypes.data_as(dp), v3.ctypes.data_as(dp),
                     s.area.ctypes.data_as(dp), s.afac, 1.0)
        t0 = time.perf_counter()
        R.ref_fill(0, rows, 0, n, buf.ctypes.data_as(dp), 3 * rows)
        t_asm = time.perf_counter() - t0
        R.ref_destroy()
    else:
        L = ob.lib()
        x, self9 = ob.incenters_and_self(s)
        t0 = time.perf_counter()
        L.orc_gr_block(n, v1.ctypes.data_as(dp), v2.ctypes.data_as(dp), v3.ctypes.data_as(dp),
                       s.area.ctypes.data_as(dp), 1.0, x.ctypes.data_as(dp), self9.ctypes.data_as(dp), 0, rows, 0, n,
                       buf.ctypes.data_as(dp), 3 * rows)
        t_asm = time.perf_counter() - t0
    from scipy.linalg import lapack
    n3 = 3 * n
    nl = min(n_lu, n3)
    rng = np.random.default_rng(seed)
    A = np.asfortranarray(rng.standard_normal((nl, nl)) + np.sqrt(nl) * np.eye(nl))
    B = np.asfortranarray(rng.standard_normal((nl, 6)))
    t0 = time.perf_counter()
    lu, piv, info = lapack.dgetrf(A, overwrite_a=1)
    t_lu = time.perf_counter() - t0
    t0 = time.perf_counter()
    lapack.dgetrs(lu, piv, B)
    t_sv = time.perf_counter() - t0
    asm = t_asm * n / rows
    fac = t_lu * (n3 / nl) ** 3
    sv = t_sv * (n3 / nl) ** 2
    parts = dict(assembly_s=asm, lu_s=fac, solve_s=sv, threads=threads, kind=kind,
                 sample=f"assembly of {rows} of {n} target rows ({'kernel.cpp' if R is not None else 'C port'}, "
                        f"OpenMP {threads} threads) scaled by pairs; dgetrf+dgetrs (OpenBLAS via scipy, "
                        f"{threads} threads) at order {nl} scaled by ({n3}/{nl})^3 and ^2")
    return asm + fac + sv, parts


def host_bytes_available():
    try:
        import psutil
        return int(psutil.virtual_memory().available)
    except Exception:
        return None


def cpu_reference_solve(tri, iarea, truearea):
    """One complete BEST solve on the host cores with the reference's own code: the reference's
    kernel.cpp assembly of every entry of GR (oracle/_ref, OpenMP over source columns; the oracle's C
    restatement, equal to it bit for bit, when _ref is absent), BEST's deflation (best.f:406-425),
    LAPACK dgetrf (best.f:444) and dgetrs for the 6 flows (besolve.f90:133; OpenBLAS via scipy, all
    host threads).  Timed part by part with a monotonic clock; then, untimed, the 5 strain flows and
    DIFCO/VISCO for the tensors.  Returns (seconds, parts, tensors)."""
    import ctypes

    from oracle import best as ob
    threads = os.cpu_count() or 1
    s = ob.setup(tri, iarea, truearea)
    n, n3 = s.n, 3 * s.n
    R = ob.ref_lib()
    dp = ctypes.POINTER(ctypes.c_double)
    t0 = time.perf_counter()
    if R is not None:
        v1, v2, v3 = s.colmajor()
        R.ref_create(n, v1.ctypes.data_as(dp), v2.ctypes.data_as(dp), v3.ctypes.data_as(dp),
                     s.area.ctypes.data_as(dp), s.afac, 1.0)
        gr = np.empty((n3, n3), dtype=np.float64, order="F")
        R.ref_fill(0, n, 0, n, gr.ctypes.data_as(dp), n3)
        x = np.empty(n3)
        R.ref_incenters(x.ctypes.data_as(dp))
        dm = R.ref_diag_mean()
        R.ref_destroy()
    else:
        gr, x, self9 = ob.assemble(s)
        dm = ob.diag_mean(self9, n)
    t1 = time.perf_counter()
    xmu, gdef = ob.deflation_vectors(s, dm)
    ob.deflate(s, gr, xmu, gdef)
    t2 = time.perf_counter()
    lu, ipiv, info = ob.getrf(gr)
    t3 = time.perf_counter()
    B6, _ = ob.getrs(lu, ipiv, ob.rhs6(x, n))
    t4 = time.perf_counter()
    V5, _ = ob.getrs(lu, ipiv, ob.strain5(x, n))
    del lu, gr
    t = ob.difco(B6, x, s.area, n)
    chip, _ = ob.visco(V5, B6, x, s.area, n, 0)
    rep = ob.report(t, chip)
    parts = dict(assembly_s=t1 - t0, deflation_s=t2 - t1, lu_s=t3 - t2, solve_s=t4 - t3, threads=threads,
                 kind="reference" if R is not None else "port", info=int(info),
                 sample=f"complete solve at N={n} (order {n3}): {'the reference kernel.cpp' if R is not None else 'the C port'}"
                        f" assembly of all {n * n} pairs (OpenMP, {threads} threads), deflation, dgetrf + dgetrs "
                        f"(OpenBLAS via scipy, {threads} threads) on that matrix; nothing scaled")
    tens = dict(D_t=rep["DTRANS"], D_r=rep["DR"], chiprime=chip, Dtt=t["Dtt"], Drr=t["Drr"], Dtr=t["Dtr"],
                urc=t["urc"], udr=t["udr"])
    return t4 - t0, parts, tens


def full_solve_fits(n):
    """Whether a complete host solve fits in host memory: GR is 72 N^2 bytes, plus room to spare."""
    avail = host_bytes_available()
    return avail is None or avail > 72.0 * n * n * 1.15 + 4e9


def run_reference(args, rank):
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    tri, ta, tv = make_mesh(args.workload)
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    # warm-up: small bounded samples (thread pools, library loading), not complete solves
    for _ in range(args.warmup):
        cpu_reference_sample(tri, w["iarea"], ta, rows=16, n_lu=1024)
    vals, parts = [], None
    if full_solve_fits(w["N"]):
        t_start = time.perf_counter()
        while len(vals) < max(1, args.steps):
            v, parts, _ = cpu_reference_solve(tri, w["iarea"], ta)
            vals.append(v)
            if time.perf_counter() - t_start + v > args.ref_budget_s:
                break
        v = float(np.median(vals))
        sample = parts["sample"]
    else:
        v, parts = cpu_reference_sample(tri, w["iarea"], ta)
        vals = [v]
        sample = ("host memory too small for a complete solve (72 N^2 bytes); " + parts["sample"])
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s",
        "n_gpus": args.gpus, "steps": len(vals), "steps_requested": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "step_s": vals,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "N": w["N"], "order": 3 * w["N"], "desc": w["desc"],
                   "warmup_kind": "bounded samples (16 assembly rows, order-1024 LU), not complete solves",
                   "budget_s": args.ref_budget_s},
        "cpu_baseline": {"value": v, "unit": "s", "cores": parts["threads"], "kind": parts["kind"],
                         "sample": sample,
                         "parts_s": {k: parts[k] for k in ("assembly_s", "deflation_s", "lu_s", "solve_s") if k in parts}},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------

def fp64_peak_tflops(torch, dev):
    """cuBLAS DGEMM 8192^3 (best of 3): the FP64 denominator (MEASURED_PEAKS.json has none)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def tensors_of(solver, x, st, bh):
    """D_t, D_r traces and CHI' (proportional to [eta]) from an 11-RHS solve with the current factors
    (untimed): best/difco.f on the 6 flows, best/visco.f on the 5 strain flows."""
    B = solver.solve(np.hstack([bh.rhs6(x), bh.strain5(x)]))
    t = bh.difco(x, st.area, B[:, :6])
    chip, _ = bh.visco(x, st.area, B[:, 6:], B[:, :6])
    tr = bh.traces(t)
    return dict(D_t=tr["DTRANS"], D_r=tr["DR"], chiprime=chip, Dtt=t["Dtt"], Drr=t["Drr"], Dtr=t["Dtr"],
                urc=t["urc"], udr=t["udr"])


# ---- DRAM traffic of the tcgen05 GEMM over the LU's launches (profiles/tc_gemm_traffic_lu_shapes.md)
def lu_gemm_shapes(n3, leaf=128):
    """The (m, n, k) of every GEMM of the mixed LU's recursion at order n3, in launch order (a replay
    of MixedSolver's rlu / trsm recursion: 2,017 launches at n3 = 61,440; a triangular solve 256 deep
    is one 256-deep leaf, without a GEMM)."""
    out = []

    def split(sz):
        return max((sz // 2) // leaf * leaf, leaf)

    def trsm_left(h, w):
        if h <= 2 * leaf or w <= 0:
            return
        h1 = split(h)
        trsm_left(h1, w)
        out.append((h - h1, w, h1))
        trsm_left(h - h1, w)

    def trsm_right(h, m):
        if h <= 2 * leaf or m <= 0:
            return
        h1 = split(h)
        trsm_right(h1, m)
        out.append((m, h - h1, h1))
        trsm_right(h - h1, m)

    def rlu(sz):
        if sz <= leaf:
            return
        h = split(sz)
        r = sz - h
        rlu(h)
        trsm_left(h, r)
        trsm_right(h, r)
        out.append((r, r, h))
        rlu(r)

    rlu(n3)
    return out


def gemm_algorithmic_bytes(m, n, k):
    """BF16 operands read once, the FP32 C read and written once."""
    return 2 * (m * k + k * n) + 8 * m * n


# DRAM bytes / algorithmic bytes of single k_gemm_bf16_tc launches, from ncu captures on B200
# (dram__bytes_read.sum + dram__bytes_write.sum; profiles/tc_gemm_traffic_lu_shapes.md)
GEMM_TRAFFIC_RATIO = {
    "k<=256": 23675392 / gemm_algorithmic_bytes(128, 30720, 128),
    "k<=2048": (190902784 + 65673472) / gemm_algorithmic_bytes(1024, 30720, 1024),
    "square>=8192": (1338633472 + 251912448) / gemm_algorithmic_bytes(8192, 8192, 8192),
    "k>2048": (2286619392 + 1036582144) / gemm_algorithmic_bytes(16384, 16384, 4096),
}


def panel_update(m, n, k):
    """The products the LU runs on the TF32 panel kernel (k_panel_tf32, mixed.cu): K = 128 with one
    side at most 128, or at most 256 with the other at most 3,840; every other product runs on the
    BF16 tcgen05 GEMM."""
    return k == 128 and (min(m, n) <= 128 or (min(m, n) <= 256 and max(m, n) <= 3840))


def gemm_traffic_per_launch(n3):
    """(estimated DRAM bytes, algorithmic bytes, launches) per tcgen05 GEMM launch of one
    factorisation at order n3: each launch's algorithmic bytes times the measured ratio of its shape
    class."""
    shapes = [sh for sh in lu_gemm_shapes(n3) if not panel_update(*sh)]
    alg = traffic = 0.0
    for m, n, k in shapes:
        a = gemm_algorithmic_bytes(m, n, k)
        if k <= 256:
            r = GEMM_TRAFFIC_RATIO["k<=256"]
        elif k <= 2048:
            r = GEMM_TRAFFIC_RATIO["k<=2048"]
        elif min(m, n, k) >= 8192:
            r = GEMM_TRAFFIC_RATIO["square>=8192"]
        else:
            r = GEMM_TRAFFIC_RATIO["k>2048"]
        alg += a
        traffic += a * r
    return traffic / len(shapes), alg / len(shapes), len(shapes)


def tensor_errors(got, want):
    """Relative differences of BEST's results: D_t, D_r traces and CHI' ([eta] is proportional); the
    full D_tt, D_rr tensors; D_tr relative to sqrt(|D_tt| |D_rr|); the centres of resistance and
    diffusion relative to the body's size (the largest of the two centres' and 1 A)."""
    out = {"D_t": relerr(got["D_t"], want["D_t"]), "D_r": relerr(got["D_r"], want["D_r"]),
           "eta": relerr(got["chiprime"], want["chiprime"]), "Dtt_tensor": relerr(got["Dtt"], want["Dtt"]),
           "Drr_tensor": relerr(got["Drr"], want["Drr"])}
    if "Dtr" in got and "Dtr" in want:
        sc = np.sqrt(np.max(np.abs(want["Dtt"])) * np.max(np.abs(want["Drr"])))
        out["Dtr_tensor"] = float(np.max(np.abs(np.asarray(got["Dtr"]) - want["Dtr"])) / sc)
    for k in ("urc", "udr"):
        if k in got and k in want:
            sc = max(1.0, float(np.max(np.abs(want[k]))))
            out[k] = float(np.max(np.abs(np.asarray(got[k]) - want[k])) / sc)
    return out


def relerr(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def max_over_ranks(v, dist=None, device="cpu"):
    """The largest v over the ranks of the default process group (v itself without one): every rank
    times its own replica, and the job is as fast as its slowest rank."""
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seconds(ms_per_solve, world):
    """Whole-job seconds per solve when each of `world` ranks solves its own replica: the slowest
    rank's time per solve divided by the number of solves done at once (aggregate throughput)."""
    return ms_per_solve / 1e3 / world


def run_ours(args, rank, world, local_rank):
    import torch
    import best_hydro_b200 as bh

    t_start = time.perf_counter()

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    w = WORKLOADS[args.workload]
    tri, ta, tv = make_mesh(args.workload)
    st = bh.Setup(tri, w["iarea"], ta)
    n, n3 = st.n, 3 * st.n
    peaks, peak_src = load_peaks()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    modes = {"fp64": bh.BGPU_FP64, "mixed": bh.BGPU_MIXED}

    solver = bh.BhmSolver()
    solver.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = solver.incenters()
    dm = solver.diag_mean()
    xmu, gdef = st.deflation(dm)
    b0 = torch.from_numpy(bh.rhs6(x)).T.contiguous().to(dev)  # rows = right-hand sides: column-major 3n x 6
    b = torch.empty_like(b0)
    s = torch.cuda.ExternalStream(bh.lib().bgpu_stream(), device=dev)

    def step(prec):
        solver.build(eps=1e-10, direct=1 if prec == "fp64" else 0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        with torch.cuda.stream(s):
            b.copy_(b0)
        solver.solve_device(b.data_ptr(), 6, n3)

    def timed(prec, warmup, steps, stats_kernel=None, clocks=False):
        """Device ms per solve (CUDA events on the library's stream, L2 flushed before each step)."""
        bh.set_precision(modes[prec])
        for _ in range(warmup):
            step(prec)
        torch.cuda.synchronize()
        if stats_kernel is not None:
            bh.kernel_stats(stats_kernel, enable=1)
        sampler = ClockSampler(local_rank) if clocks else None
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        ev, stages = [], []
        launches0 = bh.launch_count()
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            step(prec)
            e1.record(s)
            ev.append((e0, e1))
            stages.append(bh.timings())
        torch.cuda.synchronize()
        launches = bh.launch_count() - launches0
        clk = sampler.stop() if sampler else None
        step_ms = [a.elapsed_time(c) for a, c in ev]
        kst = bh.kernel_stats(stats_kernel, enable=0) if stats_kernel is not None else None
        ms = max_over_ranks(sum(step_ms) / len(step_ms), dist, dev)
        st_ms = {k: round(float(np.mean([d[k] for d in stages])), 3) for k in ("assemble", "factor", "solve")}
        return dict(ms=ms, step_ms=step_ms, launches=launches, clocks=clk, kstats=kst, stages_ms=st_ms,
                    refine_iters=stages[-1]["refine_iters"], relres=stages[-1]["relres"])

    head = args.precision
    head_kernel = bh.BGPU_KERNEL_TC_GEMM if head == "mixed" else bh.BGPU_KERNEL_LU_GEMM64
    H = timed(head, args.warmup, args.steps, stats_kernel=head_kernel, clocks=True)
    timeline = [ln.split("; ", 1)[1] for ln in bh.log_lines() if "factorisation timeline" in ln]
    acc_head = tensors_of(solver, x, st, bh)

    # the plain FP64 path beside the mixed one: its time per solve and its tensors (the reference
    # for the mixed path's errors)
    F = acc_fp64 = None
    if head == "mixed" and not args.no_fp64:
        F = timed("fp64", 1, max(1, min(args.steps, 2)))
        acc_fp64 = tensors_of(solver, x, st, bh)

    # e2e through the C ABI with host buffers (create ... solve, copies included)
    bh.set_precision(modes[head])
    e2e = []
    h2d = 8 * (12 * n + 3 * n + len(gdef)) + (4 * n if st.ndef > 1 else 0) + 8 * 6 * n3
    d2h = 8 * (4 * n + 1 + 6 * n3)
    B_host = bh.rhs6(x)
    phases = []
    for _ in range(0 if args.no_e2e else max(1, args.steps)):
        solver.destroy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        t1 = time.perf_counter()
        xe = solver.incenters()
        dme = solver.diag_mean()
        xmu_e, gdef_e = st.deflation(dme)
        t2 = time.perf_counter()
        solver.build(eps=1e-10, direct=1 if head == "fp64" else 0, ndef=st.ndef, gdef=gdef_e, comp=st.icomp,
                     xmu=xmu_e)
        t3 = time.perf_counter()
        solver.solve(B_host)
        t4 = time.perf_counter()
        e2e.append(t4 - t0)
        phases.append((t1 - t0, t2 - t1, t3 - t2, t4 - t3))
    e2e_s = max_over_ranks(float(np.median(e2e)), dist, dev) if e2e else float("nan")
    e2e_phases = ({k: round(1e3 * float(np.median([p[i] for p in phases])), 2)
                   for i, k in enumerate(("create", "incenters_deflation", "build", "solve"))} if phases else None)
    host_notes = [ln for ln in bh.log_lines() if "host side" in ln][-2:]

    # the other workloads' records (GPU), with the headline's buffers released first
    solver.destroy()
    del b, b0
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    records = None
    if rank == 0 and world == 1 and not args.no_records and args.workload == "star_f32":
        records = collect_records(args, local_rank, t_start)

    cpu = cpu_tens = None
    if rank == 0 and world == 1 and not args.no_cpu:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        if full_solve_fits(n):
            v, parts, cpu_tens = cpu_reference_solve(tri, w["iarea"], ta)
            sample = parts["sample"]
        else:
            v, parts = cpu_reference_sample(tri, w["iarea"], ta)
            sample = "host memory too small for a complete solve (72 N^2 bytes); " + parts["sample"]
        cpu = {"value": v, "unit": "s", "cores": parts["threads"], "kind": parts["kind"], "sample": sample,
               "parts_s": {k: parts[k] for k in ("assembly_s", "deflation_s", "lu_s", "solve_s") if k in parts}}

    if rank == 0:
        gl, gms, gflop = H["kstats"]
        achieved = (gflop / max(gl, 1)) / (gms / max(gl, 1) * 1e-3) / 1e12 if gl else None
        if head == "mixed":
            peak = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
            tr_bytes, alg_bytes, nshapes = gemm_traffic_per_launch(n3)
            roof = {"kernel": "k_gemm_bf16_tc (tcgen05.mma kind::f16, TMA, TMEM accumulators): every update of "
                              "the mixed LU", "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": (achieved / peak) if achieved else None, "traffic": tr_bytes,
                    "traffic_algorithmic": alg_bytes,
                    "peak_source": f"{peak_src} bf16 sustained (MEASURED_PEAKS.json; the GEMM runs inside a long step)",
                    "traffic_note": f"DRAM bytes per launch, averaged over the factorisation's {nshapes} launches: each "
                                    "launch's algorithmic bytes (BF16 A, B read once, FP32 C read and written) times "
                                    "the DRAM/algorithmic ratio ncu measured for its shape class "
                                    "(profiles/tc_gemm_traffic_lu_shapes.md)"}
        else:
            p64 = fp64_peak_tflops(torch, dev)
            roof = {"kernel": "FP64 LU trailing-update GEMM (mma.sync f64, k_dgemm_nn_minus)", "bound": "tensor",
                    "achieved": achieved, "peak": p64, "unit": "TFLOP/s", "frac": (achieved / p64) if achieved else None,
                    "traffic": None,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)"}
        roof.update(launches_per_step=gl / max(args.steps, 1), share_of_step=gms / max(sum(H["step_ms"]), 1e-9))
        accuracy = None
        if acc_fp64 is not None or cpu_tens is not None:
            accuracy = {"refine_iterations": H["refine_iters"], "relres": H["relres"]}
            if cpu_tens is not None:
                accuracy["vs"] = ("the reference's CPU solve at this size (kernel.cpp assembly + LAPACK dgetrf/"
                                  "dgetrs, DIFCO/VISCO; cpu_baseline), 11 RHS")
                accuracy[head] = tensor_errors(acc_head, cpu_tens)
                accuracy[head]["bar"] = 1e-8 if head == "mixed" else 1e-10
                if acc_fp64 is not None:
                    accuracy["fp64"] = tensor_errors(acc_fp64, cpu_tens)
                    accuracy["fp64"]["bar"] = 1e-10
            if acc_fp64 is not None:
                accuracy["mixed_vs_fp64_gpu"] = tensor_errors(acc_head, acc_fp64)
        line = {
            "metric": METRIC,
            "value": replica_seconds(H["ms"], world), "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": H["ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head == "fp64" else "bf16 LU (f32 accumulate) + f64 refinement", "data": "synthetic",
            "config": {"workload": args.workload, "N": n, "order": n3, "desc": w["desc"], "precision": head,
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "flushed (256 MB write) between timed steps; GR is 72 N^2 bytes, far above L2",
                       "stages_ms": H["stages_ms"], "factor_timeline": timeline[-1] if timeline else None,
                       "e2e_phases_ms": e2e_phases,
                       "e2e_host_notes": host_notes},
            "roofline": roof,
            "clocks": H["clocks"],
            "e2e": {"value": replica_seconds(1e3 * e2e_s, world), "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": H["launches"],
            "fp64_path": None if F is None else {"value": F["ms"] / 1e3, "unit": "s", "steps": len(F["step_ms"]),
                                                 "warmup": 1, "stages_ms": F["stages_ms"],
                                                 "speedup_mixed_vs_fp64": F["ms"] / H["ms"]},
            "accuracy": accuracy,
            "result": {"D_t_cm2_s": acc_head["D_t"], "D_r_1_s": acc_head["D_r"], "chiprime": acc_head["chiprime"]},
            "cpu_baseline": cpu,
            "records": records,
            "peaks": {"source": peak_src, "hbm_gbs": peaks.get("hbm_gbs"), "bf16_tflops": peaks.get("bf16_tflops"),
                      "bf16_tflops_sustained": peaks.get("bf16_tflops_sustained")},
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def adjoint_record(steps, warmup, fd_vertices=64, fit_steps=20, freq=16):
    """The differentiation workload: adjoint gradients of D_t, D_r and [eta] (CHI') with respect to
    every vertex coordinate, timed; checked against central differences (h = 1e-4 A) on fd_vertices
    random vertices (seed 2); then a fit_steps-step descent on vertex normal displacements that
    brings D_t 3% below its initial value (mesh's own area, BEST's -na, for the fit)."""
    import torch
    import best_hydro_b200 as bh
    from best_hydro_b200 import meshes

    verts, faces, ta, tv = meshes.ellipsoid_vf(freq)
    nv = len(verts)

    def forward(vx, iarea):
        st = bh.Setup(meshes.to_triangles(vx, faces), iarea, ta)
        s = bh.BhmSolver()
        s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        x = s.incenters()
        xmu, gdef = st.deflation(s.diag_mean())
        s.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        B = s.solve(np.hstack([bh.rhs6(x), bh.strain5(x)]))
        tr = bh.traces(bh.difco(x, st.area, B[:, :6]))
        chip, _ = bh.visco(x, st.area, B[:, 6:], B[:, :6])
        return np.array([tr["DTRANS"], tr["DR"], chip]), s

    bh.set_precision(bh.BGPU_FP64)
    for _ in range(max(1, warmup)):
        forward(verts, 1)[1].gradient(iarea=1, truearea=ta)
    t_fwd, t_grad = [], []
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        v0, s = forward(verts, 1)
        t1 = time.perf_counter()
        vals, g = s.gradient(iarea=1, truearea=ta)
        t2 = time.perf_counter()
        t_fwd.append(t1 - t0)
        t_grad.append(t2 - t1)
    gv = meshes.corner_to_vertex(g, faces, nv)
    # central differences on random vertices
    rng = np.random.default_rng(2)
    picks = rng.choice(nv, fd_vertices, replace=False)
    h = 1e-4
    scale = np.abs(gv).reshape(3, -1).max(axis=1)
    worst = np.zeros(3)
    t0 = time.perf_counter()
    for v in picks:
        for c in range(3):
            vp, vm = verts.copy(), verts.copy()
            vp[v, c] += h
            vm[v, c] -= h
            fd = (forward(vp, 1)[0] - forward(vm, 1)[0]) / (2 * h)
            worst = np.maximum(worst, np.abs(fd - gv[:, v, c]) / scale)
    t_fd = time.perf_counter() - t0
    history = []
    sdisp = np.zeros(nv)
    if fit_steps:
        # descent on normal displacements s_i (v_i + s_i n_i, n_i the outward unit normal at the vertex)
        nrm = np.zeros_like(verts)
        for f in faces:
            e = np.cross(verts[f[1]] - verts[f[0]], verts[f[2]] - verts[f[0]])
            nrm[f] += e
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        d0 = forward(verts, 0)[0][0]
        target = 0.97 * d0
        for it in range(fit_steps):
            vals_k, sk = forward(verts + sdisp[:, None] * nrm, 0)
            _, gk = sk.gradient(iarea=0)
            gs = (meshes.corner_to_vertex(gk, faces, nv)[0] * nrm).sum(axis=1)  # dD_t / ds_i
            r = (vals_k[0] - target) / target
            history.append(float(r))
            # steepest descent on r^2 / 2 with the step that zeroes the linearised residual
            sdisp -= (r * target) * gs / float(gs @ gs)
    bh.set_precision(-1)
    return {
        "value": float(np.median(t_grad)), "unit": "s", "steps": steps, "warmup": warmup,
        "N": len(faces), "vertices": nv, "forward_solve_s": float(np.median(t_fwd)),
        "values": {"D_t": vals[0], "D_r": vals[1], "chiprime": vals[2]},
        "fd_check": {"vertices": fd_vertices, "seed": 2, "h_A": h, "worst_abs_err_over_max_grad": worst.tolist(),
                     "seconds": t_fd},
        "fit": {"target": "D_t 3% below initial (mesh's own area)", "relative_residual_per_step": history,
                "max_normal_displacement_A": float(np.abs(sdisp).max())},
        "log": [ln for ln in bh.log_lines() if ln.startswith("gradient")][-1:],
    }


def run_adjoint(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    w = WORKLOADS[args.workload]
    rec = adjoint_record(args.steps, args.warmup, freq=w["gen"][1])
    line = {
        "metric": "s per adjoint gradient (D_t, D_r, [eta] w.r.t. 3 x 2562 vertex coordinates)",
        "value": rec["value"], "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": rec["value"] * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "N": rec["N"], "vertices": rec["vertices"], "desc": w["desc"]},
    }
    line.update({k: rec[k] for k in ("forward_solve_s", "values", "fd_check", "fit", "log")})
    if rank == 0:
        print(json.dumps(line), flush=True)


SERIES_FREQS = (11, 12, 14, 16, 18, 20, 22, 23)


def series_record(steps, warmup, local_rank=0, sequential_passes=1):
    """The series workload: every mesh assembled, factored (FP64) and solved for 11 right-hand sides
    through bgpu_series_* (one CUDA graph per build), against the same meshes solved one after the
    other through the single-mesh seam; results and their 1/N extrapolation."""
    import torch
    import best_hydro_b200 as bh
    from best_hydro_b200 import meshes

    setups = []
    for f in SERIES_FREQS:
        tri, ta, tv = meshes.ellipsoid(f)
        setups.append(bh.Setup(tri, 1, ta))
    bh.set_precision(bh.BGPU_FP64)
    S = bh.Series()
    S.create(setups)
    xs = S.incenters()
    defl = []
    for st, dm in zip(setups, S.diag_means()):
        xmu, gdef = st.deflation(dm)
        defl.append((st.ndef, gdef, st.icomp, xmu))
    rhs = [np.hstack([bh.rhs6(x), bh.strain5(x)]) for x in xs]
    S.build(defl, tune=1)  # tuning pass + first graph build (warm-up)
    tune_ms = S.timings()["tune"]
    for _ in range(max(0, warmup - 1)):
        S.build(defl)
    launches0 = bh.launch_count()
    sampler = ClockSampler(local_rank)
    sampler.start()
    times = []
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S.build(defl)
        sols = S.solve(rhs)
        times.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    launches = bh.launch_count() - launches0
    dev_ms = S.timings()
    # the same meshes one after the other through the single-mesh seam
    seq, seq_sols = [], []
    for k in range(sequential_passes):
        t0 = time.perf_counter()
        out = []
        for st in setups:
            s1 = bh.BhmSolver()
            s1.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
            x = s1.incenters()
            xmu, gdef = st.deflation(s1.diag_mean())
            s1.build(eps=1e-10, direct=1, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
            out.append(s1.solve(np.hstack([bh.rhs6(x), bh.strain5(x)])))
            s1.destroy()
        seq.append(time.perf_counter() - t0)
        seq_sols = out
    same = all(np.array_equal(a.view(np.int64), b.view(np.int64)) for a, b in zip(sols, seq_sols))

    def results(solutions):
        out = []
        for st, x, B in zip(setups, xs, solutions):
            tr = bh.traces(bh.difco(x, st.area, B[:, :6]))
            chip, _ = bh.visco(x, st.area, B[:, 6:], B[:, :6])
            out.append(dict(N=st.n, D_t=tr["DTRANS"], D_r=tr["DR"], chiprime=chip))
        return out

    per = results(sols)
    ns = [d["N"] for d in per]
    ext = {k: bh.extrapolate(ns, [d[k] for d in per])[0] for k in ("D_t", "D_r", "chiprime")}
    v = float(np.median(times))
    S.destroy()
    # the same series with every mesh's factorisation on the tensor cores, side by side
    mixed = None
    try:
        M = bh.Series()
        M.create(setups)
        M.set_precision(bh.BGPU_MIXED)
        M.build(defl)  # warm-up: allocations and graph captures
        mt = []
        for _ in range(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            M.build(defl)
            msols = M.solve(rhs)
            mt.append(time.perf_counter() - t0)
        mdev = M.timings()
        mper = results(msols)
        mext = {k: bh.extrapolate(ns, [d[k] for d in mper])[0] for k in ("D_t", "D_r", "chiprime")}
        errs = {k: max(abs(a[k] / b[k] - 1) for a, b in zip(mper, per)) for k in ("D_t", "D_r", "chiprime")}
        mv = float(np.median(mt))
        mixed = {"value": mv, "unit": "s", "device_ms": {"build": mdev["build"], "solve": mdev["solve"]},
                 "speedup_vs_sequential": float(np.median(seq)) / mv,
                 "max_rel_err_vs_fp64_per_mesh": errs,
                 "extrapolated_rel_err_vs_fp64": {k: abs(mext[k] / ext[k] - 1) for k in ext},
                 "log": [ln for ln in bh.log_lines() if "series" in ln][-1:]}
        M.destroy()
    except Exception as e:
        mixed = {"error": f"{type(e).__name__}: {e}"}
    bh.set_precision(-1)
    return {
        "value": v, "unit": "s", "steps": steps, "warmup": warmup, "N": ns,
        "device_ms": {"build_graph": dev_ms["build"], "solve": dev_ms["solve"], "tuning_pass": tune_ms},
        "sequential_single_solves_s": float(np.median(seq)), "speedup_vs_sequential": float(np.median(seq)) / v,
        "bitwise_equal_to_single_solves": bool(same), "clocks": clocks, "gpu_launches": launches,
        "per_mesh": per, "extrapolated_1_over_N": ext, "autotune": bh.autotune_table(), "mixed_series": mixed,
    }


def run_series(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    w = WORKLOADS[args.workload]
    rec = series_record(args.steps, args.warmup, local_rank, sequential_passes=max(1, min(args.steps, 2)))
    line = {
        "metric": "s per series solve (8 meshes: assemble + FP64 LU + 11 RHS each)", "value": rec["value"],
        "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": rec["value"] * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "N": rec["N"], "desc": w["desc"]},
    }
    line.update({k: rec[k] for k in rec if k not in ("value", "unit", "steps", "warmup", "N")})
    if rank == 0:
        print(json.dumps(line), flush=True)


def star45_record(warmup=1, steps=1, fp64=True):
    """The precision workload at N = 40,500 (order 121,500): the mixed path's device seconds per solve
    (build + 6-RHS solve) and, with fp64, the plain FP64 path's on the same matrix and the relative
    differences of D_t, D_r, CHI' and the tensors between the two (11-RHS solves)."""
    import torch
    import best_hydro_b200 as bh

    tri, ta, tv = make_mesh("star_f45")
    st = bh.Setup(tri, WORKLOADS["star_f45"]["iarea"], ta)
    s = bh.BhmSolver()
    s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
    x = s.incenters()
    xmu, gdef = st.deflation(s.diag_mean())
    rhs6 = bh.rhs6(x)
    out, acc = {}, {}
    legs = (("mixed", bh.BGPU_MIXED, warmup, steps),) + ((("fp64", bh.BGPU_FP64, 0, 1),) if fp64 else ())
    for name, prec, w, k in legs:
        bh.set_precision(prec)
        ts = []
        for it in range(w + k):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.build(eps=1e-10, direct=1 if prec == bh.BGPU_FP64 else 0, ndef=st.ndef, gdef=gdef, comp=st.icomp,
                    xmu=xmu)
            s.solve(rhs6)
            if it >= w:
                ts.append(time.perf_counter() - t0)
        stages = bh.timings()
        acc[name] = tensors_of(s, x, st, bh)
        out[name] = {"value": float(np.median(ts)), "unit": "s", "steps": k, "warmup": w,
                     "stages_ms": {kk: round(float(stages[kk]), 2) for kk in ("assemble", "factor", "solve")},
                     "note": "host wall time of bhm_build + bhm_solve (6 RHS, host buffers)"}
    bh.set_precision(-1)
    s.destroy()
    rec = {"N": st.n, "order": 3 * st.n, "legs": out}
    if fp64:
        rec["accuracy_mixed_vs_fp64"] = tensor_errors(acc["mixed"], acc["fp64"])
        rec["speedup_mixed_vs_fp64"] = out["fp64"]["value"] / out["mixed"]["value"]
    return rec


def hmatrix_record(big=64, small=32, eps=1e-4):
    """The path for meshes beyond HBM: the star body at geodesic frequency `big` (64: N = 81,920, order
    245,760, whose dense FP64 GR would need 483 GB) through BEST's seam, where bhm_build takes the
    H-matrix path by itself; and at `small` (32: the headline mesh), where the dense paths also run,
    the H-matrix results against the mixed dense path's, at eps = 1e-4 (BEST's default -he accuracy) and
    at 1e-7 (at most 120 terms a block), against the dense paths' 1e-8 bar.
    Host wall time of bhm_build + bhm_solve (6 RHS, host buffers); the 11-RHS solve for the tensors is
    untimed."""
    import torch
    import best_hydro_b200 as bh
    from best_hydro_b200 import meshes

    rec = {"eps": eps}
    legs = ((small, bh.BGPU_HMATRIX, eps, 90), (small, bh.BGPU_HMATRIX, 1e-7, 120), (small, bh.BGPU_MIXED, eps, 90),
            (big, -1, eps, 90))
    for f, prec, leps, kmax in legs:
        tri, ta, tv = meshes.star(f)
        st = bh.Setup(tri, 0, ta)
        s = bh.BhmSolver()
        s.create(st.v1, st.v2, st.v3, st.area, st.afac, 1.0)
        x = s.incenters()
        xmu, gdef = st.deflation(s.diag_mean())
        bh.set_precision(prec)
        bh.hmatrix_set_options(128, 2.0, kmax)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.build(eps=leps, direct=0, ndef=st.ndef, gdef=gdef, comp=st.icomp, xmu=xmu)
        t1 = time.perf_counter()
        s.solve(bh.rhs6(x))
        t2 = time.perf_counter()
        bh.set_precision(-1)
        bh.hmatrix_set_options()
        path = {0: "fp64", 1: "mixed", 2: "hmatrix"}[bh.lib().bgpu_precision()]
        leg = {"N": st.n, "order": 3 * st.n, "path": path, "build_s": t1 - t0, "solve_s": t2 - t1,
               "value": t2 - t0, "unit": "s", "dense_fp64_gb": 72.0 * st.n * st.n / 1e9}
        if path == "hmatrix":
            hs = bh.hmatrix_stats()
            leg["hmatrix"] = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in hs.items()}
            leg["stored_gb"] = 8 * (hs["dense_entries"] + hs["lowrank_entries"]) / 1e9
        t = tensors_of(s, x, st, bh)
        leg.update(D_t=t["D_t"], D_r=t["D_r"], chiprime=t["chiprime"], eps=leps, kmax=kmax)
        rec[f"f{f}_{path}" + ("" if leps == eps else f"_eps{leps:.0e}")] = (leg, t)
        s.destroy()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    out = {k: v[0] for k, v in rec.items() if k != "eps"}
    mx = rec.get(f"f{small}_mixed")
    for key in (f"f{small}_hmatrix", f"f{small}_hmatrix_eps1e-07"):
        if rec.get(key) and mx:
            out[f"accuracy_{key}_vs_mixed"] = tensor_errors(rec[key][1], mx[1])
    out["eps"] = eps
    return out


def collect_records(args, local_rank, t_start):
    """The other workloads' records in the default run (each guarded; skipped past the time budget)."""
    import torch

    recs = {}
    for name, fn in (("ellipsoid_series", lambda: series_record(1, 1, local_rank)),
                     ("ellipsoid_adjoint", lambda: adjoint_record(1, 1, fd_vertices=4, fit_steps=0)),
                     ("star_f45", lambda: star45_record()),
                     ("star_f64_hmatrix", lambda: hmatrix_record())):
        if time.perf_counter() - t_start > args.records_budget_s:
            recs[name] = {"skipped": f"bench time budget of {args.records_budget_s:.0f} s reached"}
            continue
        try:
            t0 = time.perf_counter()
            recs[name] = fn()
            recs[name]["record_wall_s"] = time.perf_counter() - t0
        except Exception as e:  # a record must never cost the headline line
            recs[name] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return recs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="star_f32", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="the timed path (mixed: its FP64 comparison runs beside it)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-records", action="store_true",
                    help="skip the records of the series, adjoint and N = 40,500 workloads in the default run")
    ap.add_argument("--records-budget-s", type=float, default=600.0,
                    help="start no further record once the run has taken this many seconds")
    ap.add_argument("--ref-budget-s", type=float, default=420.0,
                    help="--impl reference: run complete solves until this many seconds would be exceeded")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if WORKLOADS[args.workload]["gen"][0] == "series":
        run_series(args, rank, world, local_rank)
        return
    if WORKLOADS[args.workload]["gen"][0] == "adjoint":
        run_adjoint(args, rank, world, local_rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
