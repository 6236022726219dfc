"""Shared test helpers: golden fixtures, synthetic meshes, and BEST's call sequence through the C ABI
(best/besolve.f90:149-240 HMPREP, then DIFCO's 6-flow solve, best/difco.f:28-49)."""
import gzip
import io
import json
import os

import numpy as np

from oracle import best as ob

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_mesh(name):
    with gzip.open(os.path.join(GOLDEN, "meshes", name + ".txt.gz"), "rt") as fh:
        text = fh.read()
    path = io.StringIO(text)
    head = path.readline().split()
    nar = int(float(head[0]))
    ta = float(head[1]) if len(head) > 1 else None
    tv = float(head[2]) if len(head) > 2 else None
    tri = np.loadtxt(path, dtype=np.float64, max_rows=nar).reshape(nar, 9)
    return tri, ta, tv


def expected_cases():
    with open(os.path.join(GOLDEN, "expected_best.json")) as fh:
        return json.load(fh)


def value_for_label(rep, label):
    return {"1/3 Trace DTT(EXACT)": rep["DTRANS"], "1/3 Trace DRR(EXACT)": rep["DR"], "CHI": rep.get("CHI"),
            "ETA (cm^3/g)": rep.get("ETA")}.get(label)


def run_gpu(solver, tri, truearea, iarea=1, cg=1.0, direct=1, eps=1e-4, ivisco=0, icov=0, truevol=None, wm=None):
    """BEST's sequence through the seam: create, incenters, diag_mean, deflation vectors computed by
    the caller, build, solve for the 6 flows (and the 5 strain flows with ivisco).  The
    post-processing (DIFCO/VISCO/OUTPUT) is the oracle's restatement, as BEST keeps its own."""
    s = ob.setup(tri, iarea, truearea)
    v1, v2, v3 = s.colmajor()
    solver.create(v1, v2, v3, s.area, s.afac, cg)
    x = solver.incenters()
    dm = solver.diag_mean()
    xmu, gdef = ob.deflation_vectors(s, dm)
    solver.build(eps=eps, direct=direct, ndef=s.ndef, gdef=gdef, comp=s.icomp, xmu=xmu)
    B6 = solver.solve(ob.rhs6(x, s.n))
    t = ob.difco(B6, x, s.area, s.n, cg)
    out = dict(setup=s, x=x, diagm=dm, xmu=xmu, gdef=gdef, B6=B6, tensors=t)
    chip = None
    if ivisco:
        V5 = solver.solve(ob.strain5(x, s.n))
        chip, dv = ob.visco(V5, B6, x, s.area, s.n, icov, cg)
        out.update(V5=V5, chiprime=chip, dvisc=dv)
    out["report"] = ob.report(t, chip, truevol, wm, iarea)
    return out


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
