"""Regenerates the golden fixtures in this folder from the reference tree (run in a container that
has it; the GPU box uses the committed files).

  meshes/2eu7_02562.txt.gz, meshes/1aki49_atom_01806.txt.gz
      the reference's example inputs (examples/best/), gzipped verbatim: BEST parses the decimal
      text, so the text itself is the fixture.
  expected_best.json
      the reference's end-to-end golden values (test/expected_best_*.txt: value, relative
      tolerance, .be label) with the flags each was produced with (test/run_tests.sh:19-68).
  gr_2eu7_sample.npz
      GR entries, incenters and the diagonal mean of 2eu7_02562 (area correction on, cg = 1)
      computed by the reference's own kernel.cpp (oracle/_ref): the first 96 rows and columns and
      4096 entries at seeded random positions.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT
"""
import gzip
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

# test/run_tests.sh:19-68: which expected file goes with which mesh and flags
CASES = {
    "2eu7": dict(mesh="2eu7_02562", file="expected_best_2eu7.txt", iarea=1, ivisco=1, icov=0, wm=30000.0),
    "2eu7_vc": dict(mesh="2eu7_02562", file="expected_best_2eu7_vc.txt", iarea=1, ivisco=1, icov=1, wm=30000.0),
    "2eu7_na": dict(mesh="2eu7_02562", file="expected_best_2eu7_na.txt", iarea=0, ivisco=1, icov=0, wm=30000.0),
    "two": dict(mesh="1aki49_atom_01806", file="expected_best_two.txt", iarea=1, ivisco=1, icov=0, wm=5000.0),
}


def parse_expected(path):
    rows = []
    for line in open(path):
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        val, tol, label = line.split(None, 2)
        rows.append(dict(value=float(val), tol=float(tol), label=label))
    return rows


def main(ref):
    os.makedirs(os.path.join(HERE, "meshes"), exist_ok=True)
    for m in ("2eu7_02562", "1aki49_atom_01806"):
        with open(os.path.join(ref, "examples", "best", m), "rb") as fi, \
                gzip.GzipFile(os.path.join(HERE, "meshes", m + ".txt.gz"), "wb", mtime=0) as fo:
            shutil.copyfileobj(fi, fo)
    out = {}
    for key, c in CASES.items():
        out[key] = dict(c, expected=parse_expected(os.path.join(ref, "test", c["file"])))
    with open(os.path.join(HERE, "expected_best.json"), "w") as fh:
        json.dump(out, fh, indent=1)

    from oracle import best as ob
    tri, ta, tv = ob.read_mesh(os.path.join(ref, "examples", "best", "2eu7_02562"))
    s = ob.setup(tri, 1, ta)
    gr, x, dm = ob.assemble_ref(s)
    rng = np.random.default_rng(2026)
    n3 = 3 * s.n
    ii = rng.integers(0, n3, 4096)
    jj = rng.integers(0, n3, 4096)
    np.savez_compressed(os.path.join(HERE, "gr_2eu7_sample.npz"), corner=np.asfortranarray(gr[:96, :96]),
                        ii=ii, jj=jj, vals=gr[ii, jj], x=x, diag_mean=np.float64(dm))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py REFERENCE_ROOT")
    main(sys.argv[1])
