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


def _same_browtab(mine, ref):
    """browtab equal as a set of facing blocks per cblk (the order inside a
    cblk's segment follows the reference's insertion order, which the solve
    and the update scatter do not depend on)."""
    ct = mine["cblktab"]
    seg = np.repeat(np.arange(ct.shape[0] - 1), np.diff(ct[:, 3]))
    a = np.lexsort((mine["browtab"], seg))
    b = np.lexsort((ref["browtab"], seg))
    return np.array_equal(mine["browtab"][a], ref["browtab"][b])


def _config_system(cid, which=0):
    systems, meta = M.config(cid, scale=1.0, seed=0)
    if cid == 4:
        # the batch's smallest and largest sides, and one between
        sides = [a.grid[0] for a in systems]
        order = np.argsort(sides, kind="stable")
        pick = {0: order[0], 1: order[-1], 2: order[len(order) // 2]}[which]
        return systems[int(pick)], meta["fact"]
    return systems[0], meta["fact"]


@pytest.mark.skipif(not U.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("cid,which", [(1, 0), (2, 0), (3, 0), (5, 0), (4, 0), (4, 1), (4, 2)],
                         ids=["C1_20^3", "C2_100^3", "C3_80^3_LU", "C5_60^3_LDLh", "C4_min_side", "C4_max_side",
                              "C4_mid_side"])
def test_analysis_matches_reference_at_benchmark_sizes(cid, which):
    """The structure the benchmark factorizes is the reference's: ordering,
    cblk/blok tables and browtab of the builder's analysis equal the
    reference's own analysis of each benchmark configuration's matrix at its
    full size (C2: 70 124 cblks)."""
    A, fact = _config_system(cid, which)
    ref, st = U.run_reference(A, fact, numfact=False)
    g = U.gpu_structure(A, st)
    ref.close()
    mine = _an().analyze(A)
    for k in ("permtab", "peritab", "cblktab", "bloktab"):
        assert np.array_equal(mine[k], g[k]), k
    assert _same_browtab(mine, g)


@pytest.mark.skipif(not U.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("make,fact", [(lambda: M.laplacian_7pt(20), "potrf"),
                                       (lambda: M.convdiff_upwind(14, 12, 9, 10.0), "getrf"),
                                       (lambda: M.laplacian_7pt(40, 33, 1), "potrf")],
                         ids=["lap20", "cd14x12x9", "lap2d_40x33"])
def test_saved_analysis_loads_as_the_reference_structure(make, fact, tmp_path):
    """The reference writes its analysis (its solverSave, and the ordering in
    the format of its ordering_save); the GPU layer's loader
    (pastix_gpu_analysis_load) reads the files back into the tables it hands
    to pastix_gpu_structure: the same ordering, cblks, bloks and facing blocks
    as the reference's SolverMatrix in memory."""
    A = make()
    ref, st = U.run_reference(A, fact, numfact=False)
    g = U.gpu_structure(A, st)
    ref.save_structure(tmp_path / "solvergen", tmp_path / "ordergen")
    ref.close()
    loaded = _an().load(tmp_path / "solvergen", tmp_path / "ordergen")
    for k in ("permtab", "peritab", "cblktab", "bloktab"):
        assert np.array_equal(loaded[k], g[k]), k
    assert _same_browtab(loaded, g)


def test_saved_analysis_rejects_bad_files(tmp_path):
    from pastix_b200 import gpu as G
    (tmp_path / "bad").write_text("7\n1 2 3\n")
    with pytest.raises(G.PastixGpuError):
        _an().load(tmp_path / "bad", tmp_path / "bad")
    with pytest.raises(G.PastixGpuError):
        _an().load(tmp_path / "missing", tmp_path / "missing")
