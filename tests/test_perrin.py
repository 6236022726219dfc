"""Physics check of the oracle against Perrin's analytic ellipsoid (oracle/perrin.py): the sphere
limit is Stokes-Einstein exactly, and BEST's D_t and D_r on the 30/20/12 A ellipsoid of the
ellipsoid workloads (without the normal jitter, which makes the surface no longer an ellipsoid)
approach Perrin's values as 1/N, their linear extrapolation in 1/N to within 3e-4 (BEST's own
workflow, best/best.f:154-157)."""
import math

import numpy as np

from best_hydro_b200 import meshes
from oracle import best as ob
from oracle import perrin

AXES = (30.0, 20.0, 12.0)


def test_sphere_limit_is_stokes_einstein():
    kt = perrin.KB * perrin.TEMPERATURE
    for r in (5.0, 20.0, 35.0):
        dt, dr, _, _ = perrin.perrin([r, r, r])
        assert abs(dt / (kt / (6 * math.pi * perrin.ETA * r * 1e-8)) - 1) < 1e-13
        assert abs(dr / (kt / (8 * math.pi * perrin.ETA * (r * 1e-8) ** 3)) - 1) < 1e-13


def test_prolate_limit_matches_closed_form():
    """For a prolate spheroid (a > b = c) Perrin's mean translational diffusion has the closed form
    kT / (6 pi eta a_eff), a_eff = sqrt(a^2 - b^2) / ln((a + sqrt(a^2 - b^2)) / b) (Perrin 1934): the
    elliptic integrals reduce to it."""
    a, b = 30.0, 12.0
    dt, _, _, _ = perrin.perrin([a, b, b])
    e = math.sqrt(a * a - b * b)
    a_eff = e / math.log((a + e) / b) * 1e-8
    kt = perrin.KB * perrin.TEMPERATURE
    assert abs(dt / (kt / (6 * math.pi * perrin.ETA * a_eff)) - 1) < 1e-12


def test_best_on_ellipsoid_converges_to_perrin():
    DT, DR, _, _ = perrin.perrin(AXES)
    ns, dts, drs = [], [], []
    for f in (6, 8, 10, 12):
        tri, ta, tv = meshes.ellipsoid(f, axes=AXES, jitter=0.0)
        r = ob.best_run(tri, ta, tv, iarea=1)
        ns.append(len(tri))
        dts.append(r.report["DTRANS"])
        drs.append(r.report["DR"])
    # monotone approach, 1/N-like: the error at f = 12 is below 0.5 %
    e_t = np.array(dts) / DT - 1
    e_r = np.array(drs) / DR - 1
    assert np.all(np.diff(np.abs(e_t)) < 0) and np.all(np.diff(np.abs(e_r)) < 0)
    assert abs(e_t[-1]) < 5e-3 and abs(e_r[-1]) < 5e-3
    A = np.vstack([np.ones(len(ns)), 1.0 / np.array(ns, dtype=float)]).T
    ext_t = np.linalg.lstsq(A, np.array(dts), rcond=None)[0][0]
    ext_r = np.linalg.lstsq(A, np.array(drs), rcond=None)[0][0]
    assert abs(ext_t / DT - 1) < 3e-4, ext_t / DT - 1
    assert abs(ext_r / DR - 1) < 3e-4, ext_r / DR - 1
