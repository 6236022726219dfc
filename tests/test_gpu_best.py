"""End-to-end parity of the plain FP64 path through BEST's seam (bhm_create ... bhm_solve): the
reference's golden results (test/expected_best_*.txt, 2e-4) and the oracle's tensors at 1e-10
relative (D_t, D_r, D_tr, centres of resistance/diffusion, [eta])."""
import numpy as np
import pytest

from oracle import best as ob
from best_hydro_b200 import BhmSolver, meshes
from tests.helpers import expected_cases, golden_mesh, rel, run_gpu, value_for_label

pytestmark = pytest.mark.gpu
TOL = 1e-10


def compare_to_oracle(g, o):
    """D_t, D_r at 1e-10 relative; the coupling D_tr relative to its natural scale sqrt(|Dtt| |Drr|)
    and the centres relative to the body's size (both vanish by symmetry on symmetric bodies, where a
    plain relative error would measure rounding noise)."""
    for key in ("Dtt", "Drr"):
        assert rel(g["tensors"][key], o.tensors[key]) < TOL, key
    scale = np.sqrt(np.max(np.abs(o.tensors["Dtt"])) * np.max(np.abs(o.tensors["Drr"])))
    assert np.max(np.abs(g["tensors"]["Dtr"] - o.tensors["Dtr"])) / scale < TOL, "Dtr"
    size = np.sqrt(np.mean(o.x.reshape(3, -1) ** 2) * 3)
    for key in ("urc", "udr"):
        assert np.max(np.abs(g["tensors"][key] - o.tensors[key])) / size < TOL, key
    if o.chiprime is not None:
        assert abs(g["chiprime"] / o.chiprime - 1) < TOL


@pytest.mark.parametrize("key", ["2eu7", "2eu7_vc", "2eu7_na", "two"])
def test_golden_results_through_the_seam(key):
    c = expected_cases()[key]
    tri, ta, tv = golden_mesh(c["mesh"])
    solver = BhmSolver()
    g = run_gpu(solver, tri, ta, iarea=c["iarea"], ivisco=c["ivisco"], icov=c["icov"], truevol=tv, wm=c["wm"])
    for e in c["expected"]:
        if e["label"] in ("Dx", "Dy", "Dz"):
            got = g["dvisc"]["xyz".index(e["label"][1])]
        else:
            got = value_for_label(g["report"], e["label"])
        assert abs(got - e["value"]) <= e["tol"] * abs(e["value"]), (e["label"], got, e["value"])
    o = ob.best_run(tri, ta, tv, iarea=c["iarea"], ivisco=c["ivisco"], icov=c["icov"], wm=c["wm"])
    compare_to_oracle(g, o)
    solver.destroy()


@pytest.mark.parametrize("case", ["icosphere_1280", "ellipsoid_5120"])
def test_configs_fp64_vs_oracle(case):
    if case == "icosphere_1280":
        tri, ta, tv = meshes.icosphere(3, 20.0)
    else:
        tri, ta, tv = meshes.ellipsoid(16)
    solver = BhmSolver()
    g = run_gpu(solver, tri, ta, iarea=1, ivisco=1, truevol=tv)
    o = ob.best_run(tri, ta, tv, iarea=1, ivisco=1)
    compare_to_oracle(g, o)
    print(f"\n{case}: D_t {g['report']['DTRANS']:.9e} oracle {o.report['DTRANS']:.9e}")
    solver.destroy()
