"""Regenerates hmcheck_glibc_misrounds.npz: for the reference's two example meshes, every entry of
GR (before deflation, area correction on, cg = 1) where the reference's TGETGR/kernel.cpp, which
call glibc's acos/sin/cos/log, differ from TGETGR's arithmetic with correctly rounded functions --
the GPU's exact entries.  These are the entries BEST's BEST_HMATRIX_CHECK (best/besolve.f90:245-277)
counts with this backend; tests/test_cr_parity.py shows that each lies in a triangle pair whose
block meets an argument at which glibc's result is not the correctly rounded one.

Needs only the oracle (pinned bit for bit to the reference's kernel.cpp by tests/test_oracle.py).
Usage: python tests/golden/make_hmcheck_list.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MESHES = ("2eu7_02562", "1aki49_atom_01806")


def differing_entries(name):
    from oracle import best as ob
    from tests import crshim
    from tests.helpers import golden_mesh
    tri, ta, tv = golden_mesh(name)
    s = ob.setup(tri, 1, ta)
    ref, _, _ = ob.assemble(s, 1.0)
    cr, _, _ = crshim.assemble_cr(s, 1.0)
    return np.argwhere(ref.view(np.int64) != cr.view(np.int64)).astype(np.int32), s


def main():
    out = {}
    for m in MESHES:
        d, s = differing_entries(m)
        out[m] = d
        out[m + "_order"] = np.int64(3 * s.n)
        print(f"{m}: {len(d)} of {(3 * s.n) ** 2} entries")
    np.savez_compressed(os.path.join(HERE, "hmcheck_glibc_misrounds.npz"), **out)


if __name__ == "__main__":
    main()
