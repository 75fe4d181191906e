"""Helpers shared by the tests: run the reference oracle on a system and hand
its analysis (the SolverMatrix + ordering) to the GPU layer or to the numpy
restatement."""
import numpy as np

from oracle import pastix_ref as R
from oracle.restate import sopalin_np as NP


def ref_available():
    return R.available()


def run_reference(system, fact, nthreads=1, mixed=False, numfact=True, **kw):
    s = R.RefSolver(system, fact=fact, nthreads=nthreads, mixed=mixed, **kw)
    s.analyze()
    st = s.structure()          # before numfact: flttype/factotype not set yet
    if numfact:
        s.numfact()
        st2 = s.structure()
        st["flttype"], st["factotype"] = st2["flttype"], st2["factotype"]
    return s, st


def gpu_structure(system, st):
    """Reference SolverMatrix tables -> pastix_gpu_structure() arguments."""
    cblk, blok = st["cblk"], st["blok"]
    cblktab = np.ascontiguousarray(cblk[:, [0, 1, 2, 5]])
    bloktab = np.ascontiguousarray(blok[:-1][:, [2, 3, 0, 1]])
    return dict(n=system.n, cblktab=cblktab, bloktab=bloktab, browtab=st["browtab"],
                permtab=st["perm"], peritab=st["invp"])


def layout_of(gst):
    return NP.Layout(gst["cblktab"], gst["bloktab"])


def ref_coeftab_1d(solver, st, layout):
    L, U = solver.coeftab(st)
    L1 = NP.ref2d_to_1d(layout, L, st["cblk"], st["blok"])
    U1 = NP.ref2d_to_1d(layout, U, st["cblk"], st["blok"]) if U is not None else None
    return L1, U1


def lower_mask(layout):
    """Mask of the coeftab entries that carry L (the strict upper part of the
    diagonal blocks holds scratch in the reference)."""
    m = np.ones(layout.off[-1], bool)
    for c in range(layout.cblknbr):
        w = int(layout.width[c])
        P = layout.panel(m, c)
        P[:w, :] &= np.tril(np.ones((w, w), bool))
    return m
