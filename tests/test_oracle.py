"""The numpy restatement (oracle/restate) pinned against the golden fixtures
the reference produced (tests/golden/make_golden.py) and, where the
reference has been built here, against the reference itself."""
import glob
import os

import numpy as np
import pytest

from oracle.restate import sopalin_np as NP
from pastix_b200 import matrices as M
from tests import refutil as U

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MAKERS = {
    "lap6_potrf": (lambda: M.laplacian_7pt(6), "potrf"),
    "diff8_potrf": (lambda: M.diffusion_lognormal(8, 8, 8, 1.0, np.random.default_rng(21)), "potrf"),
    "cd7x6x5_getrf": (lambda: M.convdiff_upwind(7, 6, 5, 10.0), "getrf"),
    "lap2d_34x31": (lambda: M.laplacian_7pt(34, 31, 1), "potrf"),
}


@pytest.mark.parametrize("name", sorted(MAKERS))
def test_restatement_matches_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    make, fact = MAKERS[name]
    A = make()
    lay = NP.Layout(g["cblktab"], g["bloktab"])
    L, Uc = NP.fillin(lay, A, g["permtab"], lu=(fact == "getrf"))
    npiv = NP.factorize(lay, L, Uc, fact, 2.0 ** -53 * float(g["anorm"]))
    assert npiv == int(g["npiv"])
    mask = U.lower_mask(lay) if fact == "potrf" else np.ones(lay.off[-1], bool)
    assert np.abs(L - g["L"])[mask].max() <= 1e-13 * np.abs(g["L"]).max()
    if fact == "getrf":
        assert np.abs(Uc - g["U"]).max() <= 1e-13 * np.abs(g["U"]).max()
    perm = g["permtab"]
    b = g["b"]
    bp = np.zeros_like(b)
    bp[perm] = b
    xp = np.stack([NP.solve(lay, L, Uc, fact, bp[:, r]) for r in range(b.shape[1])], axis=1)
    assert np.abs(xp[perm] - g["x"]).max() <= 1e-12 * np.abs(g["x"]).max()


@pytest.mark.skipif(not U.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("fact,make", [
    ("potrf", lambda: M.diffusion_lognormal(12, 11, 10, 1.0, np.random.default_rng(2))),
    ("getrf", lambda: M.convdiff_upwind(12, 10, 9, 10.0)),
    ("potrf", lambda: M.laplacian_7pt(24)),
])
def test_restatement_matches_reference(fact, make):
    A = make()
    ref, st = U.run_reference(A, fact)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, Ur = U.ref_coeftab_1d(ref, st, lay)
    L, Uc = NP.fillin(lay, A, g["permtab"], lu=(fact == "getrf"))
    NP.factorize(lay, L, Uc, fact, 2.0 ** -53 * ref.dparm("A_NORM"))
    mask = U.lower_mask(lay) if fact == "potrf" else np.ones(lay.off[-1], bool)
    assert np.abs(L - Lr)[mask].max() <= 1e-13 * np.abs(Lr).max()
    if fact == "getrf":
        assert np.abs(Uc - Ur).max() <= 1e-13 * np.abs(Ur).max()


def test_golden_files_present():
    assert len(glob.glob(os.path.join(GOLDEN, "*.npz"))) == len(MAKERS)
