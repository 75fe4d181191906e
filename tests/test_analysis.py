"""Host analysis (pastix_gpu_analyze_grid) is bit-exact with the reference's
ordering + symbolic factorization + reordering + blend split."""
import os

import numpy as np
import pytest

from pastix_b200 import matrices as M
from tests import refutil as U

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _an():
    from pastix_b200 import analysis
    return analysis


@pytest.mark.parametrize("name,make", [
    ("lap6_potrf", lambda: M.laplacian_7pt(6)),
    ("diff8_potrf", lambda: M.diffusion_lognormal(8, 8, 8, 1.0, np.random.default_rng(21))),
    ("cd7x6x5_getrf", lambda: M.convdiff_upwind(7, 6, 5, 10.0)),
    ("lap2d_34x31", lambda: M.laplacian_7pt(34, 31, 1)),
])
def test_analysis_matches_golden(name, make):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    st = _an().analyze(make())
    for k in ("permtab", "peritab", "cblktab", "bloktab"):
        assert np.array_equal(st[k], g[k]), k


@pytest.mark.skipif(not U.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("grid", [(6, 6, 6), (12, 12, 12), (20, 20, 20), (15, 10, 7), (40, 33, 1),
                                  (30, 30, 30), (64, 64, 1), (23, 31, 17)])
def test_analysis_matches_reference(grid):
    A = M.laplacian_7pt(*grid)
    ref, st = U.run_reference(A, "potrf", numfact=False)
    g = U.gpu_structure(A, st)
    mine = _an().analyze(A)
    for k in ("permtab", "peritab", "cblktab", "bloktab"):
        assert np.array_equal(mine[k], g[k]), k
    # browtab: same blocks facing each cblk
    ct = mine["cblktab"]
    for c in range(ct.shape[0] - 1):
        a = sorted(mine["browtab"][ct[c, 3]:ct[c + 1, 3]])
        b = sorted(g["browtab"][ct[c, 3]:ct[c + 1, 3]])
        assert a == b


@pytest.mark.skipif(not U.ref_available(), reason="reference oracle not built")
def test_analysis_matches_reference_general_pattern():
    A = M.convdiff_upwind(14, 12, 9, 10.0)
    ref, st = U.run_reference(A, "getrf", numfact=False)
    g = U.gpu_structure(A, st)
    mine = _an().analyze(A)
    for k in ("permtab", "cblktab", "bloktab"):
        assert np.array_equal(mine[k], g[k]), k


def test_analysis_rejects_bad_grid():
    from pastix_b200 import gpu as G
    A = M.laplacian_7pt(5)
    A.grid = (5, 5, 4)
    with pytest.raises(G.PastixGpuError):
        _an().analyze(A)
