"""Diagnostic runs of the GPU solver: one factorization and a few solves of a
seeded lognormal-diffusion grid, with the per-phase or per-level timings the
library prints on stderr when asked (PASTIX_GPU_SOLVE_PROFILE):

    python -m pastix_b200.diagnostics --grid 100 --solves 3 --solve-profile 1
        1: device time per solve phase
        2: the same per level
        3: the dataflow launches' per-level task times and their warp roles' waits

Prints the factorization and solve times and, with --phases, the factor's
per-level phase timeline (pastix_gpu_phase_log).  Used to make the summaries
under profiles/ (the ncu captures run the same command)."""
import argparse
import os
import sys


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--grid", type=int, default=60, help="grid side of the 3-D lognormal diffusion problem")
    ap.add_argument("--sigma", type=float, default=1.0)
    ap.add_argument("--fp64", action="store_true", help="FP64 factor (default: mixed, FP32 factor)")
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--solve-profile", default="", help="PASTIX_GPU_SOLVE_PROFILE level (1, 2 or 3)")
    ap.add_argument("--phases", action="store_true", help="print the factor's per-level phase timeline")
    a = ap.parse_args(argv)
    if a.solve_profile:
        os.environ["PASTIX_GPU_SOLVE_PROFILE"] = a.solve_profile
    import numpy as np
    from collections import defaultdict
    from . import matrices as M, analysis, gpu as G
    n = a.grid
    A = M.diffusion_lognormal(n, n, n, a.sigma, np.random.default_rng(0))
    st = analysis.analyze(A)
    s = G.Solver()
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT["potrf"])
    s.set_iparm(G.IPARM_MIXED, 0 if a.fp64 else 1)
    s.set_structure(st)
    s.set_spm(A)
    s.numfact(A.values)
    s.numfact(A.values)
    print("numfact_ms %.3f" % s.stats()["numfact_ms"], flush=True)
    if a.phases:
        lv = defaultdict(lambda: [1e30, -1e30, defaultdict(float)])
        for (strm, ph, l, t0, t1) in s.phase_log():
            e = lv[l]
            e[0] = min(e[0], t0)
            e[1] = max(e[1], t1)
            e[2][(strm, ph)] += t1 - t0
        print("level span_ms [stream,phase]=ms (phases: 0 diagonal blocks, 1 panel TRSM, 2 FMA GEMMs, "
              "3 tensor-core GEMMs)")
        for l in sorted(lv):
            e = lv[l]
            print(l, "%.4f" % (e[1] - e[0]), " ".join("%d,%d=%.4f" % (k[0], k[1], v) for k, v in sorted(e[2].items())))
    x, b = M.rhs_from_xtrue(A, 1, np.random.default_rng(1))
    for _ in range(max(1, a.solves)):
        xs = s.solve(b)
    print("solve_ms %.3f launches %d max|x - x_true| %.3e" % (s.stats()["solve_ms"], s.stats()["solve_launches"],
                                                               float(np.abs(xs - x).max())), flush=True)
    s.close()


if __name__ == "__main__":
    sys.exit(main())
