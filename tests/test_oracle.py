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


def _complex_symmetric(A):
    """The magnetic Laplacian's lower triangle taken as a complex symmetric
    (not Hermitian) matrix: the LDL^t of complex data."""
    A.mtxtype = M.PastixSymmetric
    return A


def _real_hermitian(A):
    """A Hermitian matrix with real values: the reference's LDL^h kernel is
    exact on it (its conjugation slip acts on real numbers)."""
    A.values = A.values.real.astype(np.complex128)
    return A


ORACLE_CASES = [
    ("potrf", lambda: M.diffusion_lognormal(12, 11, 10, 1.0, np.random.default_rng(2)), None),
    ("getrf", lambda: M.convdiff_upwind(12, 10, 9, 10.0), None),
    ("potrf", lambda: M.laplacian_7pt(24), None),
    ("sytrf", lambda: M.diffusion_lognormal(11, 10, 9, 1.0, np.random.default_rng(5)), None),
    ("sytrf", lambda: _complex_symmetric(M.magnetic_laplacian(10, 9, 8, 0.5, np.random.default_rng(6))), None),
    ("potrf", lambda: M.magnetic_laplacian(10, 9, 8, -0.5, np.random.default_rng(7)), None),
    ("hetrf", lambda: _real_hermitian(M.magnetic_laplacian(10, 9, 8, 0.5, np.random.default_rng(8))), None),
    ("hetrf", lambda: M.magnetic_laplacian(10, 9, 8, 0.5, np.random.default_rng(8)), "hefix"),
]


@pytest.mark.skipif(not U.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("fact,make,variant", ORACLE_CASES,
                         ids=["potrf", "getrf", "potrf24", "sytrf", "sytrf_z", "potrf_z", "hetrf_zreal",
                              "hetrf_z_fixed"])
def test_restatement_matches_reference(fact, make, variant):
    A = make()
    ref, st = U.run_reference(A, fact, variant=variant)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, Ur = U.ref_coeftab_1d(ref, st, lay)
    L, Uc = NP.fillin(lay, A, g["permtab"], lu=(fact == "getrf"))
    npiv = NP.factorize(lay, L, Uc, fact, 2.0 ** -53 * ref.dparm("A_NORM"))
    assert npiv == ref.iparm("STATIC_PIVOTING")
    mask = np.ones(lay.off[-1], bool) if fact == "getrf" else U.lower_mask(lay)
    assert np.abs(L - Lr)[mask].max() <= 1e-13 * np.abs(Lr).max()
    if fact == "getrf":
        assert np.abs(Uc - Ur).max() <= 1e-13 * np.abs(Ur).max()
    # the solve of the restatement against the reference's own solve
    x, b = M.rhs_from_xtrue(A, 2, np.random.default_rng(4))
    xr = ref.solve(b)
    perm = g["permtab"]
    bp = np.zeros_like(b)
    bp[perm] = b
    xp = np.stack([NP.solve(lay, L, Uc, fact, bp[:, r]) for r in range(2)], axis=1)
    assert np.abs(xp[perm] - xr).max() <= 1e-11 * np.abs(xr).max()
    assert np.abs(xp[perm] - x).max() <= 1e-9


@pytest.mark.skipif(not U.ref_available(), reason="reference oracle not built")
def test_reference_ldlh_conjugation_slip_on_complex_data():
    """Records the reference's LDL^h behaviour on genuinely complex Hermitian
    data (kernels/core_zhetrfsp.c:92 conjugates with increment 1 a row of
    stride lda): its factors differ from those of A and its direct solve does
    not solve A x = b, while the one-increment fix (the "hefix" build) and the
    restatement agree and solve it."""
    A = M.magnetic_laplacian(8, 7, 6, 0.5, np.random.default_rng(1))
    x, b = M.rhs_from_xtrue(A, 1, np.random.default_rng(2))
    Af = A.to_scipy_full()
    for variant, bad in ((None, True), ("hefix", False)):
        ref, st = U.run_reference(A, "hetrf", variant=variant)
        xr = ref.solve(b)
        rel = np.abs(b - Af @ xr).max() / np.abs(b).max()
        assert (rel > 1e-2) if bad else (rel < 1e-13), (variant, rel)


def test_golden_files_present():
    assert len(glob.glob(os.path.join(GOLDEN, "*.npz"))) == len(MAKERS)
