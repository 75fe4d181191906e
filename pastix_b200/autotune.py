"""Autotuner of the factorization's kernel variants and launch shapes.

The reference fixes its block sizes at compile time and ranks kernels with
offline polynomial models; here each knob of pastix_gpu_set_tuning is chosen
per problem by measuring the factorization itself (device time from the
library's CUDA events), by coordinate descent over a small candidate space:

  trsm_gemm_rows   panel height above which the TRSM runs as a GEMM
  tc_min_mn        smallest M x N update sent to the tensor cores
  la_reserved_sms  SMs the lookahead stream leaves to the critical path
  wide_panel       narrowest diagonal block given to the left-looking
                   512-thread panel kernel (0: none)
  mixed_gemm       3xFP16 vs 3xTF32 vs one TF32 product (objective "solve": the
                   refinement's extra iterations are part of the cost)

`tune` returns the chosen values and every measurement; `TuningCache`
remembers the choice per structure (n, cblknbr, bloknbr, factorization,
precision) in a JSON file.
"""
import ctypes as C
import json
import os

import numpy as np

from . import gpu as G

KNOBS = {"mixed_gemm": 0, "tc_kernel": 1, "lookahead": 2, "la_reserved_sms": 3, "trsm_gemm": 4,
         "trsm_gemm_rows": 5, "tc_min_mn": 6, "wide_panel": 7, "tc_tma": 8, "tc_pair_min": 9,
         "dmma": 10, "solve_flow": 11, "graph": 12}

DEFAULT_SPACE = {
    "trsm_gemm_rows": [128, 256, 512],
    "tc_min_mn": [4096, 8192, 16384],
    "la_reserved_sms": [0, 16, 32],
}


def _lib():
    L = G.load()
    if not hasattr(L, "_tune_ready"):
        L.pastix_gpu_set_tuning.argtypes = [C.c_void_p, C.c_int, C.c_int64]
        L.pastix_gpu_get_tuning.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L._tune_ready = True
    return L


def set_knob(solver, name, value):
    G._check("pastix_gpu_set_tuning", _lib().pastix_gpu_set_tuning(solver._h, KNOBS[name], int(value)))


def get_knob(solver, name):
    v = np.zeros(1, np.int64)
    G._check("pastix_gpu_get_tuning", _lib().pastix_gpu_get_tuning(solver._h, KNOBS[name], G._p(v)))
    return int(v[0])


def measure(solver, values, b=None, reps=2, objective="numfact"):
    """Median device time (ms) of numfact (+ solve and refinement when
    objective == "solve"), after one untimed run that rebuilds the plan."""
    solver.numfact(values)
    if objective == "solve" and b is not None:
        solver.solve_and_refine(b)
    ts = []
    for _ in range(reps):
        solver.numfact(values)
        st = solver.stats()
        t = st["numfact_ms"]
        if objective == "solve" and b is not None:
            solver.solve_and_refine(b)
            st = solver.stats()
            t += st["solve_ms"] + st["refine_ms"]
        ts.append(t)
    return float(np.median(ts))


def tune(solver, values, b=None, space=None, reps=2, objective="numfact", rounds=1, measure_fn=None):
    """Coordinate descent over `space` (knob -> candidate values).  Returns
    (best settings, best time, list of (settings, time) measured)."""
    space = dict(DEFAULT_SPACE if space is None else space)
    if objective == "solve" and "mixed_gemm" not in space:
        space["mixed_gemm"] = [3, 2, 1]
    meas = measure_fn or (lambda: measure(solver, values, b, reps, objective))
    best = {k: get_knob(solver, k) for k in space}
    for k, v in best.items():
        set_knob(solver, k, v)
    best_t = meas()
    log = [(dict(best), best_t)]
    for _ in range(rounds):
        changed = False
        for k, cands in space.items():
            for v in cands:
                if v == best[k]:
                    continue
                set_knob(solver, k, v)
                t = meas()
                trial = dict(best)
                trial[k] = v
                log.append((trial, t))
                if t < best_t:
                    best_t, best[k], changed = t, v, True
            set_knob(solver, k, best[k])
        if not changed:
            break
    return best, best_t, log


class TuningCache:
    """Chosen settings per structure, kept in a JSON file."""

    def __init__(self, path):
        self.path = path
        self.data = {}
        if os.path.exists(path):
            with open(path) as f:
                self.data = json.load(f)

    @staticmethod
    def key(struct, fact, mixed, complex_=False):
        ct = np.asarray(struct["cblktab"])
        return "n%d_c%d_b%d_%s_%s%s" % (struct["n"], ct.shape[0] - 1, np.asarray(struct["bloktab"]).shape[0],
                                        fact, "mixed" if mixed else "fp64", "_z" if complex_ else "")

    def get(self, key):
        return self.data.get(key)

    def put(self, key, settings):
        self.data[key] = settings
        with open(self.path, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)

    def apply(self, solver, key):
        s = self.get(key)
        if s:
            for k, v in s.items():
                set_knob(solver, k, v)
        return s
