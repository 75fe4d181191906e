"""Autotuner: coordinate descent and cache on the host (fake measurements),
and on the GPU the tuning knobs of the C ABI with a real measured search."""
import numpy as np
import pytest

from pastix_b200 import autotune as AT
from pastix_b200 import matrices as M


def test_coordinate_descent_finds_separable_minimum(monkeypatch):
    state = {"trsm_gemm_rows": 256, "tc_min_mn": 8192, "la_reserved_sms": 16}
    monkeypatch.setattr(AT, "set_knob", lambda s, k, v: state.__setitem__(k, v))
    monkeypatch.setattr(AT, "get_knob", lambda s, k: state[k])
    target = {"trsm_gemm_rows": 512, "tc_min_mn": 4096, "la_reserved_sms": 0}
    cost = lambda: sum(abs(np.log2(state[k] + 1) - np.log2(target[k] + 1)) for k in target) + 1.0
    best, t, log = AT.tune(None, None, measure_fn=cost, rounds=2)
    assert best == target
    assert t == pytest.approx(1.0)
    assert state == target                       # the chosen values are left set
    assert len(log) >= 1 + sum(len(v) - 1 for v in AT.DEFAULT_SPACE.values())


def test_tuning_cache_roundtrip(tmp_path):
    st = {"n": 10, "cblktab": np.zeros((4, 4)), "bloktab": np.zeros((7, 4))}
    c = AT.TuningCache(str(tmp_path / "tune.json"))
    k = AT.TuningCache.key(st, "potrf", True)
    assert c.get(k) is None
    c.put(k, {"trsm_gemm_rows": 128})
    assert AT.TuningCache(str(tmp_path / "tune.json")).get(k) == {"trsm_gemm_rows": 128}


@pytest.mark.gpu
def test_gpu_tuning_knobs_and_search():
    from pastix_b200 import analysis
    from pastix_b200 import gpu as G
    A = M.diffusion_lognormal(24, 23, 22, 1.0, np.random.default_rng(4))
    st = analysis.analyze(A)
    s = G.Solver()
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT["potrf"])
    s.set_iparm(G.IPARM_MIXED, 1)
    s.set_iparm(G.IPARM_REFINEMENT, G.REFINE["cg"])
    s.set_structure(st)
    s.set_spm(A)
    assert AT.get_knob(s, "trsm_gemm_rows") == 256
    with pytest.raises(G.PastixGpuError):
        AT.set_knob(s, "mixed_gemm", 7)
    x, b = M.rhs_from_xtrue(A, 1, np.random.default_rng(5))
    space = {"trsm_gemm_rows": [128, 256], "la_reserved_sms": [0, 16], "mixed_gemm": [3, 2, 1]}
    best, t, log = AT.tune(s, A.values, b, space=space, objective="solve")
    assert all(best[k] in v for k, v in space.items()) and t > 0 and len(log) >= 4
    for k, v in best.items():
        assert AT.get_knob(s, k) == v
    s.numfact(A.values)
    xs = s.solve_and_refine(b)
    r = b - A.to_scipy_full() @ xs
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-12
    s.close()
