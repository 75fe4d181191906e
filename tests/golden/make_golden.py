"""Generate the golden fixtures from the reference CPU path (oracle/_ref).

Run in a checkout where the reference has been built
(python oracle/refbuild/build_ref.py); writes tests/golden/*.npz:
for a few small grids, the reference's ordering and SolverMatrix tables, its
factor coeftab (1D layout) and its solution of a seeded right-hand side.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pastix_b200 import matrices as M  # noqa: E402
from tests import refutil as U  # noqa: E402

CASES = {
    "lap6_potrf": (lambda: M.laplacian_7pt(6), "potrf"),
    "diff8_potrf": (lambda: M.diffusion_lognormal(8, 8, 8, 1.0, np.random.default_rng(21)), "potrf"),
    "cd7x6x5_getrf": (lambda: M.convdiff_upwind(7, 6, 5, 10.0), "getrf"),
    "lap2d_34x31": (lambda: M.laplacian_7pt(34, 31, 1), "potrf"),
}


def main():
    for name, (make, fact) in CASES.items():
        A = make()
        ref, st = U.run_reference(A, fact)
        g = U.gpu_structure(A, st)
        lay = U.layout_of(g)
        L, Uc = U.ref_coeftab_1d(ref, st, lay)
        x, b = M.rhs_from_xtrue(A, 2, np.random.default_rng(99))
        xr = ref.solve(b)
        out = dict(cblktab=g["cblktab"], bloktab=g["bloktab"], permtab=g["permtab"], peritab=g["peritab"],
                   L=L, b=b, x=xr, anorm=ref.dparm("A_NORM"), npiv=ref.iparm("STATIC_PIVOTING"))
        if Uc is not None:
            out["U"] = Uc
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
