"""The drop-in through the reference's own API: the reference sources built
a second time with the GPU layer plugged into their factorization, solve and
refinement tables (pastix_b200/refplug/pastix_gpu_plug.c, linked with one
--wrap per plug point by oracle/refbuild/build_ref.py) run the call sequence
of example/simple.c -- pastixInit, analysis, pastix_task_numfact,
pastix_task_solve, pastix_task_refine, pastixFinalize -- and give the
solution of the unmodified reference's CPU build."""
import os
import subprocess

import numpy as np
import pytest

from oracle import pastix_ref as R
from pastix_b200 import matrices as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NTH = os.cpu_count() or 1

PLUG_POINTS = (["coeftabInit", "pastixFinalize"] +
               ["sopalin_%s%s" % (p, f) for p in "sdcz" for f in ("potrf", "getrf", "sytrf", "trsm", "diag")] +
               ["sopalin_chetrf", "sopalin_zhetrf"] +
               ["%s_%s_smp" % (p, f) for p in "dz" for f in ("grad", "gmres")])

needs_plug = pytest.mark.skipif(not (R.available() and R.available("gpuplug")),
                                reason="GPU-plugged reference build absent")


@needs_plug
def test_plugged_build_wraps_every_plug_point():
    """The plugged build defines the wrapper of every plug point and loads
    libpastix_gpu.so (no GPU needed)."""
    lib = R.LIBS["gpuplug"]
    syms = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    for p in PLUG_POINTS:
        assert (" __wrap_%s\n" % p) in syms, p
    needed = subprocess.run(["readelf", "-d", lib], capture_output=True, text=True).stdout
    assert "libpastix_gpu.so" in needed


def _simple(A, fact, variant, mixed=False, refine=None, nrhs=2, **kw):
    """example/simple.c on one instance: numfact, solve, refine."""
    x, b = M.rhs_from_xtrue(A, nrhs, np.random.default_rng(5))
    r = R.RefSolver(A, fact=fact, nthreads=NTH, mixed=mixed, refine=refine, variant=variant, **kw)
    r.analyze()
    r.numfact()
    x0 = r.solve(b)
    x1 = r.refine(b, x0) if refine else None
    out = dict(x0=x0, x1=x1, pivots=r.iparm("STATIC_PIVOTING"), iters=r.iparm("NBITER"))
    r.close()
    return out, x, b


DROPIN_CASES = [
    ("potrf", lambda: M.diffusion_lognormal(16, 15, 14, 1.0, np.random.default_rng(3)), False, "cg", None),
    ("getrf", lambda: M.convdiff_upwind(14, 13, 12, 10.0), False, "gmres", None),
    ("potrf", lambda: M.diffusion_lognormal(16, 15, 14, 1.0, np.random.default_rng(3)), True, "cg", None),
    ("getrf", lambda: M.convdiff_upwind(14, 13, 12, 10.0), True, "gmres", None),
    ("sytrf", lambda: M.diffusion_lognormal(12, 11, 10, 1.0, np.random.default_rng(4)), False, "gmres", None),
    ("hetrf", lambda: M.magnetic_laplacian(10, 9, 8, 0.5, np.random.default_rng(8)), False, "gmres", "hefix"),
]


@pytest.mark.gpu
@needs_plug
@pytest.mark.parametrize("fact,make,mixed,refine,cpu_variant", DROPIN_CASES,
                         ids=["potrf", "getrf", "potrf_mixed", "getrf_mixed", "sytrf", "hetrf_z"])
def test_reference_api_runs_on_the_gpu(fact, make, mixed, refine, cpu_variant):
    A = make()
    gpu, x, b = _simple(A, fact, "gpuplug", mixed=mixed, refine=refine)
    cpu, _, _ = _simple(A, fact, cpu_variant, mixed=mixed, refine=refine)
    scale = np.abs(cpu["x0"]).max()
    # the direct solve: FP64 factors agree with the CPU build's solve; single
    # precision factors at their own accuracy
    tol = 1e-11 if not mixed else 1e-4
    assert np.abs(gpu["x0"] - cpu["x0"]).max() <= tol * scale
    assert gpu["pivots"] == cpu["pivots"]
    # refinement through the reference's pastix_task_refine: backward error
    Af = A.to_scipy_full()
    r = b - Af @ gpu["x1"]
    assert (np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)).max() <= 1e-12
    assert np.abs(gpu["x1"] - x).max() <= 1e-9
    assert gpu["iters"] >= 0
