"""GPU parity: the CUDA factorization/solve against the reference's own CPU
path (oracle/_ref) and the numpy restatement, on the same structure and
seeded inputs.  Tolerances: FP64 factors agree to 1e-12 relative (max-norm
over the factor); FP32 (mixed) factors to 2e-6 relative against the
reference's own mixed factorization, on the FMA tiles and on the default
tensor-core path alike (measured on B200: 4.5e-7 .. 6.2e-7 with FMA tiles,
4.5e-7 .. 9.9e-7 with the split tensor-core products, up to 40^3)."""
import os
import numpy as np
import pytest

from pastix_b200 import matrices as M
from tests import refutil as U

pytestmark = pytest.mark.gpu

CASES = [
    ("lap6", lambda: M.laplacian_7pt(6), "potrf"),
    ("lap20", lambda: M.laplacian_7pt(20), "potrf"),
    ("diff14", lambda: M.diffusion_lognormal(14, 14, 14, 1.0, np.random.default_rng(3)), "potrf"),
    ("diff2d", lambda: M.diffusion_lognormal(40, 33, 1, 0.5, np.random.default_rng(4)), "potrf"),
    # tall panels (TRSM as a GEMM, diagonal-block inverses in the solve) and a root wider than 256
    ("diff26", lambda: M.diffusion_lognormal(26, 25, 24, 1.0, np.random.default_rng(12)), "potrf"),
    ("cd10", lambda: M.convdiff_upwind(10, 10, 10, 10.0), "getrf"),
    ("cd9x7x5", lambda: M.convdiff_upwind(9, 7, 5, 10.0), "getrf"),
    # LU with diagonal blocks of 128 and 256 columns (the wide-panel kernel)
    ("cd16", lambda: M.convdiff_upwind(16, 16, 16, 10.0), "getrf"),
]
# the largest sizes of each form the test budget allows (the reference runs
# on all host threads): 40^3 LL^t, 32^3 LU
LARGE = [
    ("diff40", lambda: M.diffusion_lognormal(40, 40, 40, 1.0, np.random.default_rng(13)), "potrf"),
    ("cd32", lambda: M.convdiff_upwind(32, 32, 32, 10.0), "getrf"),
]
NTH = os.cpu_count() or 1
MIXED_TOL = 2e-6


def _gpu_solver(system, st, fact, mixed=False, refine=None):
    from pastix_b200 import gpu as G
    s = G.Solver()
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT[fact])
    s.set_iparm(G.IPARM_MIXED, 1 if mixed else 0)
    if refine:
        s.set_iparm(G.IPARM_REFINEMENT, G.REFINE[refine])
    s.set_structure(U.gpu_structure(system, st))
    s.set_spm(system)
    return s


@pytest.mark.parametrize("name,make,fact", CASES + LARGE, ids=[c[0] for c in CASES + LARGE])
def test_factor_matches_reference(name, make, fact):
    A = make()
    ref, st = U.run_reference(A, fact, nthreads=NTH)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, Ur = U.ref_coeftab_1d(ref, st, lay)
    s = _gpu_solver(A, st, fact)
    s.numfact(A.values)
    if name in [c[0] for c in LARGE]:
        # the large update and TRSM GEMMs ran on the FP64 tensor cores (DMMA)
        assert s.stats()["tc_flops"] > 0.5 * s.stats()["gemm_flops"], s.stats()
    Lg, Ug = s.coeftab()
    mask = U.lower_mask(lay) if fact == "potrf" else np.ones(lay.off[-1], bool)
    scale = np.abs(Lr).max()
    assert np.abs(Lg - Lr)[mask].max() <= 1e-12 * scale
    if fact == "getrf":
        assert np.abs(Ug - Ur).max() <= 1e-12 * np.abs(Ur).max()
    ip, dp = s.params()
    assert ip[45] == ref.iparm("STATIC_PIVOTING")
    assert abs(dp[23] - ref.dparm("A_NORM")) <= 1e-12 * ref.dparm("A_NORM")


@pytest.mark.parametrize("name,make,fact", CASES, ids=[c[0] for c in CASES])
def test_solve_matches_reference(name, make, fact):
    A = make()
    ref, st = U.run_reference(A, fact)
    s = _gpu_solver(A, st, fact)
    s.numfact(A.values)
    rng = np.random.default_rng(7)
    x, b = M.rhs_from_xtrue(A, 4, rng)
    xg = s.solve(b)
    xr = ref.solve(b)
    assert np.abs(xg - xr).max() <= 1e-11 * np.abs(xr).max()
    assert np.abs(xg - x).max() <= 1e-9


@pytest.mark.parametrize("name,make,fact", [c for c in CASES if c[2] == "potrf"],
                         ids=[c[0] for c in CASES if c[2] == "potrf"])
def test_mixed_factor_matches_reference_mixed(name, make, fact, fp32_gemm):
    A = make()
    ref, st = U.run_reference(A, fact, mixed=True)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, _ = U.ref_coeftab_1d(ref, st, lay)
    assert Lr.dtype == np.float32
    s = _gpu_solver(A, st, fact, mixed=True)
    s.numfact(A.values)
    Lg, _ = s.coeftab()
    assert Lg.dtype == np.float32
    mask = U.lower_mask(lay)
    assert np.abs(Lg.astype(np.float64) - Lr)[mask].max() <= MIXED_TOL * np.abs(Lr).max()


TC_CASES = [CASES[4], ("cd20x18x16", lambda: M.convdiff_upwind(20, 18, 16, 10.0), "getrf")] + LARGE


@pytest.mark.parametrize("mode", ["default", "3xf16", "3xtf32"])
@pytest.mark.parametrize("name,make,fact", TC_CASES, ids=[c[0] for c in TC_CASES])
def test_mixed_tensor_core_factor_matches_reference_mixed(name, make, fact, mode, monkeypatch):
    """The mixed factorization with its update and TRSM GEMMs on tcgen05 with
    split products (the default mode, and each split form: 3xFP16 with per-row
    power-of-two scales, 3xTF32) against the reference's own single-precision
    factors, at the FMA path's accuracy: the splits keep the products at FP32
    accuracy."""
    if mode != "default":
        monkeypatch.setenv("PASTIX_GPU_MIXED_GEMM", mode)
    A = make()
    ref, st = U.run_reference(A, fact, mixed=True, nthreads=NTH)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, Ur = U.ref_coeftab_1d(ref, st, lay)
    s = _gpu_solver(A, st, fact, mixed=True)
    s.numfact(A.values)
    stats = s.stats()
    assert stats["tc_flops"] > 0.5 * stats["gemm_flops"], stats
    assert stats["tc_timeouts"] == 0
    Lg, Ug = s.coeftab()
    mask = U.lower_mask(lay) if fact == "potrf" else np.ones(lay.off[-1], bool)
    err = np.abs(Lg.astype(np.float64) - Lr)[mask].max() / np.abs(Lr).max()
    assert err <= MIXED_TOL, err
    if fact == "getrf":
        assert np.abs(Ug.astype(np.float64) - Ur).max() <= MIXED_TOL * np.abs(Ur).max()
    s.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_cg_refinement_reaches_1e12(mixed):
    A = M.diffusion_lognormal(16, 16, 16, 1.0, np.random.default_rng(11))
    ref, st = U.run_reference(A, "potrf", numfact=False)
    s = _gpu_solver(A, st, "potrf", mixed=mixed, refine="cg")
    s.numfact(A.values)
    rng = np.random.default_rng(5)
    x, b = M.rhs_from_xtrue(A, 2, rng)
    xs = s.solve_and_refine(b)
    Af = A.to_scipy_full()
    r = b - Af @ xs
    assert np.linalg.norm(r, axis=0).max() / np.linalg.norm(b, axis=0).min() <= 1e-12
    bwd = np.abs(r).max() / (abs(Af).sum(axis=1).max() * np.abs(xs).max() + np.abs(b).max())
    assert bwd <= 1e-12
    ip, dp = s.params()
    assert ip[52] >= (1 if mixed else 0)


@pytest.fixture
def fp32_gemm(monkeypatch):
    monkeypatch.setenv("PASTIX_GPU_MIXED_GEMM", "fp32")


@pytest.mark.parametrize("mode,tol", [("3xtf32", MIXED_TOL), ("3xf16", MIXED_TOL), ("tf32", 5e-3)])
def test_tf32_tensor_core_factor_and_refinement(mode, tol, monkeypatch):
    """The mixed factorization's large update GEMMs run on tcgen05 with TF32
    operands (one product, or the 3xTF32 split): the factor stays within that
    mode's accuracy of the reference's FP32 factor and CG refinement still
    reaches 1e-12."""
    monkeypatch.setenv("PASTIX_GPU_MIXED_GEMM", mode)
    A = M.diffusion_lognormal(26, 25, 24, 1.0, np.random.default_rng(12))
    ref, st = U.run_reference(A, "potrf", mixed=True)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, _ = U.ref_coeftab_1d(ref, st, lay)
    s = _gpu_solver(A, st, "potrf", mixed=True, refine="cg")
    s.numfact(A.values)
    stats = s.stats()
    assert stats["tc_flops"] > 0.3 * stats["gemm_flops"], stats
    assert stats["tc_timeouts"] == 0
    Lg, _ = s.coeftab()
    mask = U.lower_mask(lay)
    err = np.abs(Lg.astype(np.float64) - Lr)[mask].max() / np.abs(Lr).max()
    assert err <= tol, err
    x, b = M.rhs_from_xtrue(A, 1, np.random.default_rng(6))
    xs = s.solve_and_refine(b)
    r = b - A.to_scipy_full() @ xs
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-12


@pytest.mark.parametrize("mixed", [False, True])
def test_lu_gmres_refinement_reaches_1e12(mixed):
    """GETRF + GMRES(30) (refinement/z_refine_gmres.c) on the upwind
    convection-diffusion operator; FP32 factors use the tensor-core GEMM."""
    A = M.convdiff_upwind(18, 17, 16, 10.0)
    ref, st = U.run_reference(A, "getrf", numfact=False)
    s = _gpu_solver(A, st, "getrf", mixed=mixed, refine="gmres")
    from pastix_b200 import gpu as G
    s.set_iparm(G.IPARM_GMRES_IM, 30)
    s.numfact(A.values)
    x, b = M.rhs_from_xtrue(A, 4, np.random.default_rng(9))
    xs = s.solve_and_refine(b)
    Af = A.to_scipy_full()
    r = b - Af @ xs
    assert (np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)).max() <= 1e-12
    bwd = np.abs(r).max() / (abs(Af).sum(axis=1).max() * np.abs(xs).max() + np.abs(b).max())
    assert bwd <= 1e-12
    assert np.abs(xs - x).max() <= 1e-8


@pytest.mark.parametrize("name,make", [("cd10", lambda: M.convdiff_upwind(10, 10, 10, 10.0)),
                                       ("cd20x18x16", lambda: M.convdiff_upwind(20, 18, 16, 10.0))])
def test_mixed_lu_factor_matches_reference_mixed(name, make, fp32_gemm):
    A = make()
    ref, st = U.run_reference(A, "getrf", mixed=True)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, Ur = U.ref_coeftab_1d(ref, st, lay)
    s = _gpu_solver(A, st, "getrf", mixed=True)
    s.numfact(A.values)
    Lg, Ug = s.coeftab()
    assert np.abs(Lg.astype(np.float64) - Lr).max() <= MIXED_TOL * np.abs(Lr).max()
    assert np.abs(Ug.astype(np.float64) - Ur).max() <= MIXED_TOL * np.abs(Ur).max()


# --- LDL^t / LDL^h and complex data ------------------------------------------
def _complex_symmetric(A):
    A.mtxtype = M.PastixSymmetric
    return A


def _real_hermitian(A):
    A.values = A.values.real.astype(np.complex128)
    return A


def _complex_general(A):
    """Full storage of the magnetic Laplacian with the lower triangle scaled
    by (1 + 0.5i): a complex unsymmetric matrix with a symmetric pattern."""
    import scipy.sparse as sp
    F = A.to_scipy_full().tocoo()
    v = np.where(F.row > F.col, F.data * (1 + 0.5j), F.data)
    G = sp.csc_matrix((v, (F.row, F.col)), shape=F.shape)
    G.sort_indices()
    return M.SparseSystem(n=A.n, colptr=G.indptr.astype(np.int64), rowptr=G.indices.astype(np.int64),
                          values=G.data.copy(), mtxtype=M.PastixGeneral, grid=A.grid, name=A.name + "_gen",
                          meta={})


LDL_CASES = [
    ("sytrf", lambda: M.diffusion_lognormal(20, 19, 18, 1.0, np.random.default_rng(5)), None),
    ("sytrf", lambda: _complex_symmetric(M.magnetic_laplacian(14, 13, 12, 0.5, np.random.default_rng(6))), None),
    ("potrf", lambda: M.magnetic_laplacian(14, 13, 12, -0.5, np.random.default_rng(7)), None),
    ("hetrf", lambda: _real_hermitian(M.magnetic_laplacian(14, 13, 12, 0.5, np.random.default_rng(8))), None),
    ("hetrf", lambda: M.magnetic_laplacian(14, 13, 12, 0.5, np.random.default_rng(8)), "hefix"),
    ("getrf", lambda: _complex_general(M.magnetic_laplacian(9, 8, 7, 0.5, np.random.default_rng(9))), None),
    ("hetrf", lambda: M.magnetic_laplacian(24, 24, 24, 0.5, np.random.default_rng(8)), "hefix"),
]
LDL_IDS = ["sytrf_d", "sytrf_z", "potrf_z", "hetrf_zreal", "hetrf_z", "getrf_z", "hetrf_z24"]


@pytest.mark.parametrize("fact,make,variant", LDL_CASES, ids=LDL_IDS)
def test_ldl_and_complex_factor_solve_match_reference(fact, make, variant):
    """FP64 / complex128 factors to 1e-12 of the reference's own factors
    (LDL^h on complex data: the reference with its one-increment fix, see
    oracle/refbuild/build_ref.py), and the solve to 1e-11 of its solve."""
    A = make()
    ref, st = U.run_reference(A, fact, variant=variant, nthreads=NTH)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, Ur = U.ref_coeftab_1d(ref, st, lay)
    s = _gpu_solver(A, st, fact)
    s.numfact(A.values)
    Lg, Ug = s.coeftab()
    mask = np.ones(lay.off[-1], bool) if fact == "getrf" else U.lower_mask(lay)
    assert np.abs(Lg - Lr)[mask].max() <= 1e-12 * np.abs(Lr).max()
    if fact == "getrf":
        assert np.abs(Ug - Ur).max() <= 1e-12 * np.abs(Ur).max()
    ip, dp = s.params()
    assert ip[45] == ref.iparm("STATIC_PIVOTING")
    assert abs(dp[12] - ref.dparm("FACT_THFLOPS")) <= 1e-9 * ref.dparm("FACT_THFLOPS")
    x, b = M.rhs_from_xtrue(A, 3, np.random.default_rng(17))
    xg = s.solve(b)
    xr = ref.solve(b)
    assert np.abs(xg - xr).max() <= 1e-11 * np.abs(xr).max()
    assert np.abs(xg - x).max() <= 1e-9
    s.close()


@pytest.mark.parametrize("fact,make,variant", [LDL_CASES[0], LDL_CASES[1], LDL_CASES[4], LDL_CASES[6]],
                         ids=["sytrf_d", "sytrf_z", "hetrf_z", "hetrf_z24"])
def test_ldl_mixed_factor_matches_reference_mixed(fact, make, variant):
    """LDL^t / LDL^h in single precision (default path: the LDL updates
    C -= A D B^t run on FMA tiles) against the reference's mixed factors."""
    A = make()
    ref, st = U.run_reference(A, fact, mixed=True, variant=variant, nthreads=NTH)
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    Lr, _ = U.ref_coeftab_1d(ref, st, lay)
    s = _gpu_solver(A, st, fact, mixed=True)
    s.numfact(A.values)
    Lg, _ = s.coeftab()
    assert Lg.dtype == Lr.dtype
    mask = U.lower_mask(lay)
    assert np.abs(Lg.astype(np.complex128) - Lr)[mask].max() <= MIXED_TOL * np.abs(Lr).max()
    s.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_hetrf_gmres_refinement_reaches_1e12(mixed):
    """C5's path at a small size: LDL^h of the shifted magnetic Laplacian
    (complex Hermitian indefinite), complex GMRES(30) to ||r||/||b|| <= 1e-12."""
    A = M.magnetic_laplacian(16, 15, 14, 0.5, np.random.default_rng(10))
    ref, st = U.run_reference(A, "hetrf", numfact=False)
    s = _gpu_solver(A, st, "hetrf", mixed=mixed, refine="gmres")
    from pastix_b200 import gpu as G
    s.set_iparm(G.IPARM_GMRES_IM, 30)
    s.numfact(A.values)
    x, b = M.rhs_from_xtrue(A, 4, np.random.default_rng(11))
    xs = s.solve_and_refine(b)
    Af = A.to_scipy_full()
    r = b - Af @ xs
    assert (np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)).max() <= 1e-12
    assert np.abs(xs - x).max() <= 1e-9
    ip, _ = s.params()
    assert ip[52] <= (10 if mixed else 2)
    s.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_factorization_graph_replay_matches_direct(mixed, monkeypatch):
    """The factorization sequence (norm, fill-in, every level's panels, TRSMs
    and update GEMMs on both lookahead streams) captured once as a CUDA graph
    and replayed (PGPU_TUNE_GRAPH = 1; 0 launches kernel by kernel; the
    default, -1, captures factors of at most 2^24 coefficients, as here):
    its factors equal the directly launched ones, a new set of values reuses
    the same graph, and the per-phase timings come from its event nodes."""
    from pastix_b200 import autotune as AT
    A = M.diffusion_lognormal(24, 23, 22, 1.0, np.random.default_rng(21))
    ref, st = U.run_reference(A, "potrf", numfact=False)
    s = _gpu_solver(A, st, "potrf", mixed=mixed)
    assert AT.get_knob(s, "graph") == -1
    s.numfact(A.values)                  # (default: captured, this size)
    s.numfact(A.values)
    assert s.stats()["graph_replayed"] == 1.0
    AT.set_knob(s, "graph", 0)           # launched kernel by kernel
    s.numfact(A.values)
    assert s.stats()["graph_replayed"] == 0.0
    L0, _ = s.coeftab()
    AT.set_knob(s, "graph", 1)
    s.numfact(A.values)                  # capture
    s.numfact(A.values)                  # replay
    st_ = s.stats()
    assert st_["graph_replayed"] == 1.0
    assert st_["diag_ms"] > 0 and st_["gemm_ms"] > 0   # phase timings from the graph's event nodes
    L1, _ = s.coeftab()
    tol = 1e-12 if not mixed else 1e-5
    assert np.abs(L1.astype(np.float64) - L0).max() <= tol * np.abs(L0).max()
    vals2 = A.values * 2.0               # same pattern, new values: same graph
    s.numfact(vals2)
    L2, _ = s.coeftab()
    assert np.abs(L2.astype(np.float64) - np.sqrt(2.0) * L0).max() <= 10 * tol * np.abs(L0).max()
    x, b = M.rhs_from_xtrue(A, 2, np.random.default_rng(3))
    xs = s.solve(2.0 * b)
    assert np.abs(xs - x).max() <= (1e-9 if not mixed else 1e-3)
    s.close()


WIDE_CASES = [
    ("potrf", lambda: M.diffusion_lognormal(26, 25, 24, 1.0, np.random.default_rng(12)), False),
    ("potrf", lambda: M.diffusion_lognormal(26, 25, 24, 1.0, np.random.default_rng(12)), True),
    ("getrf", lambda: M.convdiff_upwind(16, 16, 16, 10.0), False),
    ("getrf", lambda: M.convdiff_upwind(16, 16, 16, 10.0), True),
    ("sytrf", lambda: M.diffusion_lognormal(20, 19, 18, 1.0, np.random.default_rng(5)), False),
    ("sytrf", lambda: M.diffusion_lognormal(20, 19, 18, 1.0, np.random.default_rng(5)), True),
    ("hetrf", lambda: M.magnetic_laplacian(14, 13, 12, 0.5, np.random.default_rng(8)), True),
    ("potrf", lambda: M.magnetic_laplacian(14, 13, 12, -0.5, np.random.default_rng(7)), True),
]


@pytest.mark.parametrize("fact,make,mixed", WIDE_CASES,
                         ids=["potrf_d", "potrf_s", "getrf_d", "getrf_s", "sytrf_d", "sytrf_s", "hetrf_c", "potrf_c"])
def test_wide_panel_kernel_matches_narrow(fact, make, mixed):
    """Diagonal blocks of 128 columns and more go to the left-looking
    512-thread kernel; with it switched off (PGPU_TUNE_WIDE_PANEL = 0) the
    right-looking panel kernel factorizes them.  Both factors agree to the
    rounding of their different summation orders."""
    from pastix_b200 import autotune as AT
    A = make()
    ref, st = U.run_reference(A, fact, numfact=False)
    s = _gpu_solver(A, st, fact, mixed=mixed)
    assert AT.get_knob(s, "wide_panel") == 128
    s.numfact(A.values)
    L1, U1 = s.coeftab()
    AT.set_knob(s, "wide_panel", 0)
    s.numfact(A.values)
    L0, U0 = s.coeftab()
    tol = 2e-5 if mixed else 1e-12
    g = U.gpu_structure(A, st)
    lay = U.layout_of(g)
    mask = np.ones(lay.off[-1], bool) if fact == "getrf" else U.lower_mask(lay)
    assert np.abs(L1 - L0)[mask].max() <= tol * np.abs(L0).max()
    if fact == "getrf":
        assert np.abs(U1 - U0).max() <= tol * np.abs(U0).max()
    s.close()


@pytest.mark.parametrize("fact,make", [
    ("potrf", lambda: M.diffusion_lognormal(26, 25, 24, 1.0, np.random.default_rng(12))),
    ("getrf", lambda: M.convdiff_upwind(20, 18, 16, 10.0)),
], ids=["potrf", "getrf"])
@pytest.mark.parametrize("trsm_gemm", [1, 0], ids=["trsm_gemm", "trsm_rows"])
def test_tma_operands_match_producer_split(fact, make, trsm_gemm, monkeypatch):
    """3xTF32 update and TRSM GEMMs with the operands split once per panel
    into hi / lo planes and loaded by TMA (PGPU_TUNE_TC_TMA = 1) against the
    producer warps splitting each tile (= 0): the same products, up to the
    order of the scatter-add reductions."""
    from pastix_b200 import autotune as AT
    monkeypatch.setenv("PASTIX_GPU_MIXED_GEMM", "3xtf32")   # the same arithmetic on both paths
    A = make()
    ref, st = U.run_reference(A, fact, numfact=False)
    s = _gpu_solver(A, st, fact, mixed=True)
    assert AT.get_knob(s, "tc_tma") == 1
    AT.set_knob(s, "trsm_gemm", trsm_gemm)
    AT.set_knob(s, "tc_pair_min", 0)       # every launch pairs its 128-row tiles
    s.numfact(A.values)
    L1, U1 = s.coeftab()
    AT.set_knob(s, "tc_tma", 0)
    s.numfact(A.values)
    L0, U0 = s.coeftab()
    assert np.abs(L1.astype(np.float64) - L0).max() <= 2e-6 * np.abs(L0).max()
    if fact == "getrf":
        assert np.abs(U1.astype(np.float64) - U0).max() <= 2e-6 * np.abs(U0).max()
    st_ = s.stats()
    assert st_["tc_ms"] > 0
    s.close()


DMMA_CASES = LARGE + [("sytrf20", LDL_CASES[0][1], "sytrf")]


@pytest.mark.parametrize("name,make,fact", DMMA_CASES, ids=[c[0] for c in DMMA_CASES])
def test_fp64_dmma_matches_fma_tiles(name, make, fact, monkeypatch):
    """FP64 update and TRSM GEMMs on the FP64 tensor cores (DMMA, default)
    against the FMA tiles (PGPU_TUNE_DMMA = 0): the same factors to the
    rounding of their summation orders."""
    from pastix_b200 import autotune as AT
    A = make()
    ref, st = U.run_reference(A, fact, numfact=False, nthreads=NTH)
    s = _gpu_solver(A, st, fact)
    s.numfact(A.values)
    assert s.stats()["tc_flops"] > 0
    L1, U1 = s.coeftab()
    AT.set_knob(s, "dmma", 0)
    s.numfact(A.values)
    assert s.stats()["tc_flops"] == 0
    L0, U0 = s.coeftab()
    assert np.abs(L1 - L0).max() <= 1e-13 * np.abs(L0).max()
    if fact == "getrf":
        assert np.abs(U1 - U0).max() <= 1e-13 * np.abs(U0).max()
    s.close()


# dataflow solve (runs of levels whose cblks all hold a diagonal-block
# inverse, one launch per direction) for 1, 2 and 4 right-hand sides, real
# and complex, LL^t / LU / LDL^t / LDL^h, FP64 and mixed factors
FLOW_CASES = [
    ("diff26_d1", CASES[4][1], "potrf", None, False, 1),
    ("diff26_d2", CASES[4][1], "potrf", None, False, 2),
    ("diff26_s1", CASES[4][1], "potrf", None, True, 1),
    ("diff26_s4", CASES[4][1], "potrf", None, True, 4),
    ("cd32_d1", LARGE[1][1], "getrf", None, False, 1),
    ("cd32_s2", LARGE[1][1], "getrf", None, True, 2),
    ("sytrf_d4", LDL_CASES[0][1], "sytrf", None, False, 4),
    ("hetrf_z24_1", LDL_CASES[6][1], "hetrf", "hefix", False, 1),
    ("hetrf_z24_2", LDL_CASES[6][1], "hetrf", "hefix", False, 2),
    ("hetrf_z24_s4", LDL_CASES[6][1], "hetrf", "hefix", True, 4),
]


@pytest.mark.parametrize("name,make,fact,variant,mixed,nrhs", FLOW_CASES, ids=[c[0] for c in FLOW_CASES])
def test_dataflow_solve_matches_reference(name, make, fact, variant, mixed, nrhs):
    """The dataflow solve (PGPU_TUNE_SOLVE_FLOW = 1, default) takes fewer
    launches than the per-level kernels and gives the same solution: FP64
    factors to 1e-11 of the reference's solve and 1e-12 of the per-level
    solve; single-precision factors to 1e-5 of the per-level solve (the
    summation orders differ)."""
    from pastix_b200 import autotune as AT
    A = make()
    ref, st = U.run_reference(A, fact, variant=variant, nthreads=NTH, numfact=not mixed)
    s = _gpu_solver(A, st, fact, mixed=mixed)
    s.numfact(A.values)
    x, b = M.rhs_from_xtrue(A, nrhs, np.random.default_rng(41))
    assert AT.get_knob(s, "solve_flow") == 1
    xg = s.solve(b)
    n_on = s.stats()["solve_launches"]
    AT.set_knob(s, "solve_flow", 0)
    x0 = s.solve(b)
    n_off = s.stats()["solve_launches"]
    assert n_on < n_off, (n_on, n_off)
    tol = 1e-5 if mixed else 1e-12
    assert np.abs(xg - x0).max() <= tol * np.abs(x0).max()
    if not mixed:
        xr = ref.solve(b)
        assert np.abs(xg - xr).max() <= 1e-11 * np.abs(xr).max()
    s.close()


def test_factorization_from_a_saved_analysis(tmp_path):
    """Structure handoff through files: the reference's saved analysis
    (solverSave + ordering file) loaded by pastix_gpu_analysis_load drives a
    factorization and solve equal to the reference's."""
    from pastix_b200 import analysis
    A = M.diffusion_lognormal(18, 17, 16, 1.0, np.random.default_rng(31))
    ref, st = U.run_reference(A, "potrf", nthreads=NTH)
    ref.save_structure(tmp_path / "solvergen", tmp_path / "ordergen")
    g = analysis.load(tmp_path / "solvergen", tmp_path / "ordergen")
    from pastix_b200 import gpu as G
    s = G.Solver()
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT["potrf"])
    s.set_structure(g)
    s.set_spm(A)
    s.numfact(A.values)
    lay = U.layout_of(U.gpu_structure(A, st))
    Lr, _ = U.ref_coeftab_1d(ref, st, lay)
    Lg, _ = s.coeftab()
    mask = U.lower_mask(lay)
    assert np.abs(Lg - Lr)[mask].max() <= 1e-12 * np.abs(Lr).max()
    x, b = M.rhs_from_xtrue(A, 2, np.random.default_rng(3))
    assert np.abs(s.solve(b) - ref.solve(b)).max() <= 1e-11 * np.abs(x).max()
    s.close()
    ref.close()
