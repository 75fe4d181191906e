#!/usr/bin/env python3
"""Benchmark: time-to-solution at backward error <= 1e-12 on one B200,
FP32 factorization + FP64 CG refinement ("mixed") vs the FP64 factorization.

Workload (default): 3D 7-point variable-coefficient diffusion on a 100^3 grid
(n = 1e6, SPD, face coefficients lognormal(0, 1) per edge, seeded), Cholesky,
one right-hand side b = A x_true with x_true ~ U[-1, 1].  The analysis is the
grid nested dissection of the reference (done once, not timed).  One step =
numerical factorization + solve + refinement to ||r||_2/||b||_2 <= REFINE_EPS
(1e-13, both arms: the reference's 2-norm stopping test one decade below the
target, so that the infinity-norm backward error
||b - Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf) is <= 1e-12 as well; GMRES
on the upwind LU otherwise stops with that error near 2e-12).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config 1..5] [--scale S]

Prints one JSON line (rank 0).  `value`: mixed-arm time-to-solution with the
matrix values and b already in HBM (CUDA events on the library's stream);
`e2e`: the same through the C ABI with host buffers (values, b in; x out;
pinned host memory, allocated once before the timed steps).
With --impl reference the reference's own CPU path (oracle/_ref, static
scheduler, all host cores) is timed on a bounded sample (the same problem on
a smaller grid) and scaled to the full problem by the ratio of factorization
flops; N > 1 runs independent replicas (the single-system path does not
shard), rank 0 reports the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pastix_b200 import matrices as M  # noqa: E402

METRIC = "time-to-solution at backward err <=1e-12: mixed vs FP64 factor, 1 B200"
REFINE_EPS = 1e-13
CONFIG_DESC = {
    1: "laplacian_7pt 20^3 (n=8000), LLt, CG to 1e-12, nrhs 1",
    2: "diffusion_lognormal(sigma=1) 100^3 (n=1e6), LLt, FP32 factor + FP64 CG vs FP64 factor, nrhs 1",
    3: "convdiff_upwind(Pe=10) 80^3 (n=512000), LU, GMRES(30), nrhs 4",
    4: "512 x diffusion_lognormal(sigma=0.5) 2D sides U{32..256}, LLt, nrhs 8",
    5: "magnetic_laplacian 60^3 - 0.5 I, LDLh complex, GMRES, nrhs 4",
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", type=int, default=2)
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample-scale", type=float, default=1.0)
    # skip the learned cost model's measured-time evaluation (after the timed steps)
    p.add_argument("--no-cost-model", action="store_true")
    # --arms mixed: only the mixed arm, no peak measurement (the command the
    # ncu launch lists and captures in profiles/ are taken on)
    p.add_argument("--arms", default="both", choices=["both", "mixed"])
    return p.parse_args()


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def reduce_max(pg, v, local):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda:%d" % local)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            for line in out.strip().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def errors(A, b, x, xtrue):
    Af = A.to_scipy_full()
    r = b - Af @ x
    anorm_inf = abs(Af).sum(axis=1).max()
    bwd = float(np.abs(r).max() / (anorm_inf * np.abs(x).max() + np.abs(b).max()))
    rel = float((np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)).max())
    fwd = float(np.abs(x - xtrue).max() / np.abs(xtrue).max())
    return {"backward_error": bwd, "relative_residual": rel, "forward_error": fwd}


def factor_nnz(st):
    """Entries of the factor's lower part (diagonal blocks as triangles) and of
    the diagonal blocks (the solve reads their inverses whole)."""
    cb, bl = np.asarray(st["cblktab"]), np.asarray(st["bloktab"])
    nc = cb.shape[0] - 1
    w = (cb[:nc, 1] - cb[:nc, 0] + 1).astype(np.int64)
    h = np.bincount(bl[:, 2], weights=(bl[:, 1] - bl[:, 0] + 1), minlength=nc).astype(np.int64)
    return int((h * w).sum() - (w * (w - 1) // 2).sum()), int((w * w).sum())


# DRAM bytes of the tensor-core update kernel over one factorization of the
# 100^3 lognormal diffusion problem (LL^t, 3xFP16): one-pass ncu capture of all
# 228 launches of a numfact (profiles/k_gemm_scatter_tc_tma_c2_dram.md).  About
# 82 GB of the 90 GB are the scatter-add targets' partial sums (40.8 GB of
# reductions, each target line read and written back); the operands are ~4 GB.
TC_DRAM_BYTES_100CUBE = {"read": 53332129280, "write": 37116627968, "launches": 228}


def measured_peaks():
    """HBM GB/s and dense BF16 TFLOP/s of this pool's B200s: the driver-measured
    file when present, else the earlier measurement on this pool."""
    try:
        pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return {"hbm_gbs": float(pk["hbm_gbs"]), "bf16_tflops": float(pk["bf16_tflops"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def fma_peaks():
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "pastix_b200", "lib", "libpgpu_peak.so"))
    lib.pgpu_peak_fma_tflops.restype = C.c_double
    lib.pgpu_peak_fma_tflops.argtypes = [C.c_int, C.c_int]
    out = {"fp64_fma_tflops": lib.pgpu_peak_fma_tflops(0, 20000),
           "fp32_fma_tflops": lib.pgpu_peak_fma_tflops(1, 40000)}
    # TF32 tensor-core rate of cuBLAS (fp32 matmul with TF32 allowed), 8192^3,
    # best of 10 -- the denominator for the tcgen05 TF32 update GEMM
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(8192, 8192, device="cuda")
    bm = torch.randn(8192, 8192, device="cuda")
    for _ in range(3):
        a @ bm
    best = 1e30
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ bm
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = prev
    out["tf32_cublas_tflops"] = 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12
    del a, bm
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
def run_arm(A, st, b, mixed, steps, warmup, fact, refine, segments=None):
    """One arm (mixed or FP64): device-resident timing, then e2e timing.
    segments: batch of independent systems merged into A (per-system
    refinement test)."""
    import torch
    from pastix_b200 import gpu as G
    s = G.Solver(device=torch.cuda.current_device())
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT[fact])
    s.set_iparm(G.IPARM_MIXED, 1 if mixed else 0)
    s.set_iparm(G.IPARM_REFINEMENT, G.REFINE[refine])
    s.set_dparm(G.DPARM_EPSILON_REFINEMENT, REFINE_EPS)
    s.set_structure(st)
    s.set_spm(A)
    spm_ms = s.stats()["spm_ms"]   # device-side pattern setup (fill map, permuted CSR), once per pattern
    if segments is not None:
        s.set_segments(segments)
    dev = torch.device("cuda", torch.cuda.current_device())
    d_vals = torch.from_numpy(np.ascontiguousarray(A.values)).to(dev)
    d_b = torch.from_numpy(np.asfortranarray(b).reshape(-1, order="F").copy()).to(dev)
    d_x = torch.zeros_like(d_b)
    nrhs = b.shape[1]

    def step_resident():
        s.numfact(d_vals)
        from pastix_b200.gpu import load, _p, _check
        rc = load().pastix_gpu_solve_and_refine(s._h, nrhs, _p(d_b), A.n, _p(d_x), A.n)
        _check("pastix_gpu_solve_and_refine", rc)
        st_ = s.stats()
        ip, dp = s.params()
        return st_, ip, dp

    for _ in range(warmup):
        step_resident()
    torch.cuda.synchronize()
    per = []
    launches = 0
    gemm_ms = gemm_flops = tc_ms = tc_flops = 0.0
    iters = []
    t0 = time.perf_counter()
    for _ in range(steps):
        st_, ip, dp = step_resident()
        per.append(st_["numfact_ms"] + st_["solve_ms"] + st_["refine_ms"])
        launches += int(st_["numfact_launches"] + st_["solve_launches"] + st_["refine_launches"])
        gemm_ms += st_["gemm_ms"]
        gemm_flops += st_["gemm_flops"]
        tc_ms += st_["tc_ms"]
        tc_flops += st_["tc_flops"]
        iters.append(int(ip[G.IPARM_NBITER]))
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / steps
    last = dict(st_)
    x = d_x.cpu().numpy().reshape(A.n, nrhs, order="F")
    # e2e through the C ABI with host buffers: values and b in pinned host
    # memory (allocated once, outside the timed region), x read back into a
    # pinned buffer; every step copies them in and out
    from pastix_b200.gpu import load, _p, _check
    tdt = torch.complex128 if np.iscomplexobj(A.values) else torch.float64
    h_vals = torch.empty(A.values.shape, dtype=tdt, pin_memory=True)
    h_vals.numpy()[:] = A.values
    h_b = torch.empty(A.n * nrhs, dtype=tdt, pin_memory=True)
    h_b.numpy()[:] = np.asfortranarray(b).reshape(-1, order="F")
    h_x = torch.zeros(A.n * nrhs, dtype=tdt, pin_memory=True)
    e2e = []
    for _ in range(max(1, steps)):
        t = time.perf_counter()
        s.numfact(h_vals)
        _check("pastix_gpu_solve_and_refine",
               load().pastix_gpu_solve_and_refine(s._h, nrhs, _p(h_b), A.n, _p(h_x), A.n))
        e2e.append(time.perf_counter() - t)
    xh = h_x.numpy().reshape(A.n, nrhs, order="F").copy()
    s.close()
    return {
        "device_s": float(np.median(per)) / 1e3, "device_s_all": [p / 1e3 for p in per], "wall_s": wall,
        "e2e_s": float(np.median(e2e)), "launches_per_step": launches / steps, "launches": launches,
        "gemm_ms_per_step": gemm_ms / steps, "gemm_flops_per_step": gemm_flops / steps,
        "tc_ms_per_step": tc_ms / steps, "tc_flops_per_step": tc_flops / steps,
        "refine_iters": iters[-1], "factor_ms": last["numfact_ms"], "solve_ms": last["solve_ms"],
        "refine_ms": last["refine_ms"], "diag_ms": last["diag_ms"], "trsm_ms": last["trsm_ms"],
        "fact_gflops": float(dp[G.DPARM_FACT_FLOPS]), "thflops": float(dp[G.DPARM_FACT_THFLOPS]),
        "x": x, "x_e2e": xh, "spm_ms": spm_ms, "graph_replayed": bool(last.get("graph_replayed", 0.0)),
    }


def cost_model_eval(cfg, A, st, fact, mixed_values, systems=None, structs=None, nrhs=8):
    """The learned cost model judged by measured time (after the timed
    steps): the network and the flop model are fitted on the recorded task
    timings of smaller problems of the same family, their held-out
    prediction errors compared on another size, then the factorization of
    this workload is timed with its level launches ordered by each model's
    per-cblk cost and in plain cblk order; for the batch of independent
    systems the LPT shards of 8 ranks chosen by each model are also run one
    after the other and their makespans compared."""
    from pastix_b200 import costmodel as CM
    from pastix_b200 import gpu as G
    fam = {1: (2, 0.3, 0.4, 0.35), 2: (2, 0.3, 0.4, 0.35), 3: (3, 0.2, 0.25, 0.22), 5: (5, 0.25, 0.3, 0.27)}
    if cfg == 4:
        rng = np.random.default_rng(11)
        train = [M.diffusion_lognormal(int(q), int(q), 1, 0.5, rng) for q in rng.integers(32, 257, 48)]
        test = [M.diffusion_lognormal(int(q), int(q), 1, 0.5, rng) for q in rng.integers(32, 257, 16)]
    else:
        c0, s1, s2, s3 = fam[cfg]
        train = M.config(c0, scale=s1, seed=5)[0] + M.config(c0, scale=s2, seed=6)[0]
        test = M.config(c0, scale=s3, seed=7)[0]
    mixed = True
    mlp, flop = CM.train_models(train, fact, mixed)
    e_mlp, e_flop = CM.heldout_errors([mlp, flop], test, fact, mixed)
    out = {"train": "recorded task timings of %d %s" % (len(train), "2D systems" if cfg == 4 else "smaller grids"),
           "heldout_median_abs_log_err": {"mlp": e_mlp, "flop_model": e_flop}}
    # level-launch order inside the factorization of this workload
    s = G.Solver(device=0)
    s.set_iparm(G.IPARM_FACTORIZATION, G.FACT[fact])
    s.set_iparm(G.IPARM_MIXED, 1)
    s.set_structure(st)
    s.set_spm(A)
    s.numfact(mixed_values)
    esz = 4 * (2 if np.iscomplexobj(A.values) else 1)
    cplx = np.iscomplexobj(A.values)
    # (the recorded plan: real single-precision LL^t / LU updates on the tensor cores)
    info = CM.plan_tasks(st, fact, esz, use_tc=not cplx and fact in ("potrf", "getrf"), complex_=cplx)
    nc = st["cblktab"].shape[0] - 1
    out["numfact_ms"] = {
        "cblk_order": CM.numfact_ms_with_priority(s, None, mixed_values),
        "mlp_priority": CM.numfact_ms_with_priority(s, CM.cblk_costs(info, mlp.predict(info), nc), mixed_values),
        "flop_priority": CM.numfact_ms_with_priority(s, CM.cblk_costs(info, flop.predict(info), nc), mixed_values)}
    s.close()
    if cfg == 4 and systems is not None:
        from pastix_b200 import batch as B
        c_mlp = CM.system_costs(structs, mlp, fact, 4, use_tc=True)
        c_flop = np.array([B.system_flops(t) for t in structs])
        p_mlp, _ = B.shard(c_mlp, 8)
        p_flop, _ = B.shard(c_flop, 8)
        m_mlp, t_mlp = CM.shard_makespan_ms(systems, structs, p_mlp, fact, True, nrhs)
        m_flop, t_flop = CM.shard_makespan_ms(systems, structs, p_flop, fact, True, nrhs)
        out["lpt_8_shards_ms"] = {"mlp": {"makespan": m_mlp, "shards": t_mlp},
                                  "flop_model": {"makespan": m_flop, "shards": t_flop},
                                  "how": "each rank's shard (numfact + solve + CG) run on this GPU in turn"}
    mlp.close()
    return out


def errors_batch(systems, offs, b, x, xtrue):
    """Largest per-system errors of a batch (each system's own norms)."""
    out = {}
    for i, A in enumerate(systems):
        sl = slice(int(offs[i]), int(offs[i + 1]))
        e = errors(A, b[sl], x[sl], xtrue[sl])
        for k, v in e.items():
            out[k] = max(out.get(k, 0.0), v)
    return out


def cpu_reference_batch(systems, nrhs, fact, refine, mixed, nthreads, budget_s, total_flops):
    """Reference CPU path on the batch, one system after the other (the
    reference has no batched entry point), on the leading systems until
    budget_s of CPU time; scaled to the whole batch by factorization flops."""
    from oracle import pastix_ref as R
    t_sum = f_sum = 0.0
    worst = {}
    k = 0
    for A in systems:
        xs, bs = M.rhs_from_xtrue(A, nrhs, np.random.default_rng(1))
        r = R.RefSolver(A, fact=fact, nthreads=nthreads, mixed=mixed, refine=refine, eps_refine=REFINE_EPS)
        r.analyze()
        t = time.perf_counter()
        r.numfact()
        x0 = r.solve(bs)
        x1 = r.refine(bs, x0)
        t_sum += time.perf_counter() - t
        f_sum += r.dparm("FACT_THFLOPS")
        for kk, v in errors(A, bs, x1, xs).items():
            worst[kk] = max(worst.get(kk, 0.0), v)
        r.close()
        k += 1
        if t_sum >= budget_s:
            break
    return t_sum * total_flops / f_sum, k, t_sum, worst


def cpu_reference_sample(cfg, scale, sample_scale, fact, refine, mixed, steps, warmup, nthreads):
    """Reference CPU path on the same problem at `sample_scale` of the grid,
    scaled to the full problem by the factorization-flop ratio."""
    from oracle import pastix_ref as R
    systems, _ = M.config(cfg, scale=scale * sample_scale, seed=0)
    As = systems[0]
    rng = np.random.default_rng(1)
    xs, bs = M.rhs_from_xtrue(As, 1, rng)
    r = R.RefSolver(As, fact=fact, nthreads=nthreads, mixed=mixed, refine=refine, eps_refine=REFINE_EPS)
    r.analyze()
    times = []
    for i in range(warmup + steps):
        t = time.perf_counter()
        r.numfact()
        x0 = r.solve(bs)
        x1 = r.refine(bs, x0)
        dt = time.perf_counter() - t
        if i >= warmup:
            times.append(dt)
    thf = r.dparm("FACT_THFLOPS")
    err = errors(As, bs, x1, xs)
    r.close()
    return float(np.median(times)), thf, As.grid, err


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args)
    cfg = args.config
    fact = {1: "potrf", 2: "potrf", 3: "getrf", 4: "potrf", 5: "hetrf"}[cfg]
    refine = {1: "cg", 2: "cg", 3: "gmres", 4: "cg", 5: "gmres"}[cfg]
    systems, meta = M.config(cfg, scale=args.scale, seed=0)
    nrhs = meta["nrhs"] if cfg != 2 else 1
    batch = (cfg == 4)
    segments = None
    if batch:
        # 512 independent systems: this rank's longest-processing-time shard
        # (flop-count cost), merged into one block-diagonal forest
        from pastix_b200 import analysis, batch as B
        all_structs = [analysis.analyze(a) for a in systems]
        costs = [B.system_flops(t) for t in all_structs]
        parts, load = B.shard(costs, world)
        mine = parts[rank]
        bsys = [systems[i] for i in mine]
        bstructs = [all_structs[i] for i in mine]
        st_batch, segments = B.merge_structures(bstructs)
        A = B.merge_systems(bsys)
        xs_l, bs_l = zip(*[M.rhs_from_xtrue(a, nrhs, np.random.default_rng(1000 + int(i)))
                           for a, i in zip(bsys, mine)])
        xtrue, b = np.asfortranarray(np.vstack(xs_l)), np.asfortranarray(np.vstack(bs_l))
        total_flops = float(sum(costs))
    else:
        A = systems[0]
        rng = np.random.default_rng(1)
        xtrue, b = M.rhs_from_xtrue(A, nrhs, rng)
    config = {"workload": CONFIG_DESC[cfg] + ("" if args.scale == 1.0 else " scaled %.2f" % args.scale),
              "grid": list(A.grid) if not batch else "512 2D grids, sides %d..%d" % (
                  min(a.grid[0] for a in systems), max(a.grid[0] for a in systems)),
              "n": A.n, "nnz": A.nnz, "nrhs": int(b.shape[1]),
              "ordering": "reference grid nested dissection (pastixOrderGrid; Scotch unavailable)",
              "l2": "inputs larger than L2 (coeftab > 126 MB), no flush",
              "refine": "%s, stop at ||r||_2/||b||_2 <= %g" % (refine.upper(), REFINE_EPS),
              "parallelism": ("systems sharded over %d GPUs (LPT on flops)" % world if batch else "replicas")
              if world > 1 else "1 GPU"}
    if batch:
        config["systems_this_rank"] = len(mine)
        config["batch"] = "all systems of a rank merged into one forest: one launch per elimination-tree level"

    if args.impl == "reference":
        if rank != 0:
            return
        nth = os.cpu_count() or 1
        if batch:
            value, k, t_s, err = cpu_reference_batch(systems, nrhs, fact, refine, True, nth, 20.0, total_flops)
            line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "s", "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
                    "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
                    "dtype": "f32 factor + f64 refine", "data": "synthetic (seeded)", "config": config,
                    "cpu_baseline": {"value": value, "unit": "s", "cores": nth, "kind": "reference",
                                     "sample": "reference CPU mixed path, system after system: %d of %d systems "
                                               "took %.2f s, scaled to all by factorization flops" % (
                                                   k, len(systems), t_s), "errors": err},
                    "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line))
            return
        t, thf_s, grid_s, err = cpu_reference_sample(cfg, args.scale, args.cpu_sample_scale, fact, refine, True,
                                                     args.steps, args.warmup, nth)
        value, how = t, "measured on the full problem"
        if args.cpu_sample_scale != 1.0:
            # full-problem flops from the reference's own analysis (DPARM_FACT_THFLOPS)
            from oracle import pastix_ref as R
            rf = R.RefSolver(A, fact=fact, nthreads=nth)
            rf.analyze()
            thf_full = rf.dparm("FACT_THFLOPS")
            rf.close()
            value = t * thf_full / thf_s
            how = "measured %.2f s on a %s grid, scaled by factorization flops %.3e/%.3e" % (
                t, "x".join(map(str, grid_s)), thf_full, thf_s)
        line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 factor + f64 refine",
                "data": "synthetic (seeded)", "config": config,
                "cpu_baseline": {"value": value, "unit": "s", "cores": nth, "kind": "reference",
                                 "sample": "reference CPU mixed path (IPARM_MIXED=1, %s to %g; static scheduler, "
                                           "%d threads, sequential OpenBLAS), numfact+solve+refine per step, "
                                           "median of %d steps, %s" % (refine.upper(), REFINE_EPS, nth, args.steps, how),
                                 "errors": err},
                "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local)
    from pastix_b200 import analysis
    t_an = time.perf_counter()
    st = st_batch if batch else analysis.analyze(A)
    t_an = time.perf_counter() - t_an
    if args.arms == "mixed":
        mixed = run_arm(A, st, b, True, args.steps, args.warmup, fact, refine, segments)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "arms": "mixed", "value": mixed["device_s"], "unit": "s",
                              "e2e_s": mixed["e2e_s"], "factor_ms": mixed["factor_ms"], "solve_ms": mixed["solve_ms"],
                              "refine_ms": mixed["refine_ms"], "refine_iters": mixed["refine_iters"],
                              "tc_ms": mixed["tc_ms_per_step"], "config": config}))
        return
    peaks = fma_peaks() if rank == 0 else {}
    barrier(pg)
    with ClockSampler(local) as clk:
        mixed = run_arm(A, st, b, True, args.steps, args.warmup, fact, refine, segments)
        fp64 = run_arm(A, st, b, False, args.steps, args.warmup, fact, refine, segments)
    barrier(pg)
    value = reduce_max(pg, mixed["device_s"], local)
    e2e_v = reduce_max(pg, mixed["e2e_s"], local)
    fp64_v = reduce_max(pg, fp64["device_s"], local)
    if rank != 0:
        return
    if batch:
        err_m = errors_batch(bsys, segments, b, mixed["x"], xtrue)
        err_d = errors_batch(bsys, segments, b, fp64["x"], xtrue)
        err_e = errors_batch(bsys, segments, b, mixed["x_e2e"], xtrue)
    else:
        err_m = errors(A, b, mixed["x"], xtrue)
        err_d = errors(A, b, fp64["x"], xtrue)
        err_e = errors(A, b, mixed["x_e2e"], xtrue)
    g_ach = mixed["gemm_flops_per_step"] / (mixed["gemm_ms_per_step"] * 1e-3) / 1e12
    tc_ach = (mixed["tc_flops_per_step"] / (mixed["tc_ms_per_step"] * 1e-3) / 1e12
              if mixed["tc_ms_per_step"] > 0 else None)
    peak_tf32 = peaks.get("tf32_cublas_tflops")
    mp = measured_peaks()
    bf16_peak = mp["bf16_tflops"]
    # solve: algorithmic bytes of one FP32 solve -- the factor read twice (forward, backward) and
    # the right-hand side in and out in FP64 -- over the measured solve time; the diagonal blocks'
    # inverses, read whole instead of their triangles, are reported apart
    nnz_l, nnz_diag = factor_nnz(st) if not batch else (None, None)
    solve_bytes = (2 * nnz_l * 4 + 2 * A.n * nrhs * 8) if nnz_l else None
    # (at most: every diagonal block read whole, w^2 instead of w (w + 1) / 2, in both sweeps)
    inv_extra = (nnz_diag - A.n) * 4 if nnz_diag else None
    g64 = fp64["gemm_flops_per_step"] / (fp64["gemm_ms_per_step"] * 1e-3) / 1e12
    peak64 = peaks.get("fp64_fma_tflops")
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "strong" if batch else "weak", "vs_baseline": None, "dtype": "f32 factor + f64 refine", "data": "synthetic (seeded)",
        "config": config,
        "fp64": {"value": fp64_v, "unit": "s", "e2e_s": fp64["e2e_s"], "factor_ms": fp64["factor_ms"],
                 "solve_ms": fp64["solve_ms"], "refine_ms": fp64["refine_ms"], "refine_iters": fp64["refine_iters"],
                 "fact_gflops": fp64["fact_gflops"], "errors": err_d,
                 "roofline_gemm": {"bound": "fp64 fma", "achieved": g64, "peak": peak64, "unit": "TFLOP/s",
                                   "frac": g64 / peak64 if peak64 else None,
                                   "peak_source": "measured FP64 FMA microbenchmark (pastix_b200/csrc/peak.cu)"}},
        "mixed": {"factor_ms": mixed["factor_ms"], "solve_ms": mixed["solve_ms"], "refine_ms": mixed["refine_ms"],
                  "diag_ms": mixed["diag_ms"], "trsm_ms": mixed["trsm_ms"], "gemm_ms": mixed["gemm_ms_per_step"],
                  "refine_iters": mixed["refine_iters"], "fact_gflops": mixed["fact_gflops"], "errors": err_m,
                  "wall_s": mixed["wall_s"], "device_s_all": mixed["device_s_all"]},
        "mixed_speedup_vs_fp64": fp64_v / value,
        # the mixed solution against the FP64 arm's (which the GPU parity tests hold to 1e-11 of the
        # reference's own solve)
        "forward_error_vs_fp64": float(np.abs(mixed["x"] - fp64["x"]).max() / np.abs(fp64["x"]).max()),
        "roofline_solve": ({"bound": "hbm", "kernel": "one FP32 supernodal solve (forward + backward; "
                                                       "k_solve_flow on the levels with inverses)",
                            "achieved": solve_bytes / (mixed["solve_ms"] * 1e-3) / 1e9, "peak": mp["hbm_gbs"],
                            "unit": "GB/s",
                            "frac": solve_bytes / (mixed["solve_ms"] * 1e-3) / 1e9 / mp["hbm_gbs"],
                            "peak_source": mp["source"], "algorithmic_bytes": solve_bytes, "nnz_l": nnz_l,
                            "inverse_extra_bytes": inv_extra, "solve_ms": mixed["solve_ms"]}
                           if solve_bytes else None),
        "roofline": {"bound": "tensor",
                     "kernel": "k_gemm_scatter_tc_tma<3xFP16> (tcgen05 kind::f16 update + TRSM GEMM, "
                               "scatter-add epilogue)",
                     "achieved": tc_ach, "peak": bf16_peak, "unit": "TFLOP/s",
                     "frac": tc_ach / bf16_peak if (bf16_peak and tc_ach) else None,
                     # DRAM bytes per step of the kernel (ncu capture of this workload; other
                     # configurations were not captured)
                     "traffic": (TC_DRAM_BYTES_100CUBE["read"] + TC_DRAM_BYTES_100CUBE["write"]) if cfg == 2 else None,
                     "traffic_rate_gbs": ((TC_DRAM_BYTES_100CUBE["read"] + TC_DRAM_BYTES_100CUBE["write"]) /
                                          (mixed["tc_ms_per_step"] * 1e-3) / 1e9)
                                         if (cfg == 2 and mixed["tc_ms_per_step"]) else None,
                     "peak_source": "dense BF16/FP16 tensor rate, %s (%s)" % (
                         mp["source"], "MEASURED_PEAKS.json" if mp["source"] == "measured" else
                         "no MEASURED_PEAKS.json: the earlier measurement on this pool"),
                     # 3xFP16: three FP16 MMAs (lo.hi, hi.lo, hi.hi) per algorithmic product
                     "issued_frac": 3 * tc_ach / bf16_peak if (bf16_peak and tc_ach) else None,
                     "tf32_cublas_tflops": peak_tf32,
                     "algorithmic_flops_per_step": mixed["tc_flops_per_step"],
                     "tc_ms_per_step": mixed["tc_ms_per_step"],
                     "all_gemm": {"achieved": g_ach, "algorithmic_flops_per_step": mixed["gemm_flops_per_step"],
                                  "ms_per_step": mixed["gemm_ms_per_step"]}},
        "e2e": {"value": e2e_v, "unit": "s", "h2d_bytes_per_step": int(A.values.nbytes + b.nbytes),
                "d2h_bytes_per_step": int(b.nbytes), "errors": err_e},
        "gpu_launches": int(mixed["launches"]),
        "factor_graph_replayed": mixed["graph_replayed"],
        "spm_setup_ms": mixed["spm_ms"],
        "analysis_s": t_an, "peaks": peaks,
    }
    line["clocks"] = clk.summary()
    if not args.no_cost_model:
        try:
            line["cost_model"] = cost_model_eval(cfg, A, st, fact, A.values, systems if batch else None,
                                                 all_structs if batch else None, nrhs)
        except Exception as e:
            line["cost_model"] = {"error": str(e)}
    if world == 1 and not args.no_cpu_baseline and batch:
        nth = os.cpu_count() or 1
        v, k, t_s, err = cpu_reference_batch(systems, nrhs, fact, refine, True, nth, 20.0, total_flops)
        line["cpu_baseline"] = {"value": v, "unit": "s", "cores": nth, "kind": "reference",
                                "sample": "reference CPU mixed path, system after system: %d of %d systems took "
                                          "%.2f s, scaled to all by factorization flops" % (k, len(systems), t_s),
                                "errors": err}
    elif world == 1 and not args.no_cpu_baseline:
        try:
            nth = os.cpu_count() or 1
            t, thf_s, grid_s, err = cpu_reference_sample(cfg, args.scale, args.cpu_sample_scale, fact, refine,
                                                         True, 1, 0, nth)
            v, how = t, "one run of the full problem"
            if args.cpu_sample_scale != 1.0:
                v = t * mixed["thflops"] / thf_s
                how = "%.2f s on a %s grid scaled by factorization flops %.3e/%.3e" % (
                    t, "x".join(map(str, grid_s)), mixed["thflops"], thf_s)
            line["cpu_baseline"] = {"value": v, "unit": "s", "cores": nth, "kind": "reference",
                                    "sample": "reference CPU mixed path (IPARM_MIXED=1, %s to %g; static "
                                              "scheduler, %d threads, sequential OpenBLAS), numfact+solve+refine, "
                                              "%s" % (refine.upper(), REFINE_EPS, nth, how),
                                    "errors": err}
        except Exception as e:  # the oracle may be absent on a fresh checkout
            line["cpu_baseline"] = {"value": None, "unit": "s", "cores": os.cpu_count(), "kind": "reference",
                                    "sample": "unavailable: %s" % e}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
