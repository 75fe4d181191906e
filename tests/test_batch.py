"""Batch of independent systems (the 512-system configuration) merged into
one block-diagonal forest, and its sharding over ranks.

CPU tests: the merged structure factorized by the numpy restatement gives,
system by system, the factors of the separate runs; longest-processing-time
sharding; a world-size-2 gloo run in which each rank solves its shard and
rank 0 gathers every system's solution.  GPU tests: the merged batch through
the C ABI against the separate solves, and the per-system refinement test."""
import os
import socket

import numpy as np
import pytest

from oracle.restate import sopalin_np as NP
from pastix_b200 import analysis
from pastix_b200 import batch as B
from pastix_b200 import matrices as M


def _systems(k=5, seed=3):
    rng = np.random.default_rng(seed)
    sides = rng.integers(5, 13, k)
    return [M.diffusion_lognormal(int(q), int(q) + 1, 1, 0.5, rng) for q in sides]


def _factor_solve_np(struct, system, b):
    lay = NP.Layout(struct["cblktab"], struct["bloktab"])
    L, _ = NP.fillin(lay, system, struct["permtab"])
    NP.factorize(lay, L, None, "potrf", 0.0)
    bp = np.zeros_like(b)
    bp[struct["permtab"]] = b
    xp = np.stack([NP.solve(lay, L, None, "potrf", bp[:, r]) for r in range(b.shape[1])], axis=1)
    return L, xp[struct["permtab"]]


def test_merged_structure_factors_match_separate_runs():
    systems = _systems()
    structs = [analysis.analyze(s) for s in systems]
    st, offs = B.merge_structures(structs)
    A = B.merge_systems(systems)
    assert A.n == sum(s.n for s in systems) and offs[-1] == A.n
    assert st["cblktab"].shape[0] == sum(t["cblktab"].shape[0] - 1 for t in structs) + 1
    assert st["cblktab"][-1, 2] == st["bloktab"].shape[0]
    bl = [M.rhs_from_xtrue(s, 2, np.random.default_rng(7 + i)) for i, s in enumerate(systems)]
    b = np.vstack([t[1] for t in bl])
    Lm, xm = _factor_solve_np(st, A, b)
    off = 0
    for i, (s, t) in enumerate(zip(systems, structs)):
        Ls, xs = _factor_solve_np(t, s, bl[i][1])
        assert np.array_equal(Lm[off:off + Ls.size], Ls)
        off += Ls.size
        assert np.abs(xm[offs[i]:offs[i + 1]] - xs).max() <= 1e-14 * np.abs(xs).max()
        assert np.abs(xs - bl[i][0]).max() <= 1e-10


def test_lpt_shard_covers_every_system_once_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(0, 1.5, 97)
    for nr in (1, 2, 3, 8):
        parts, load = B.shard(costs, nr)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(costs)))
        assert np.allclose([costs[p].sum() for p in parts], load)
        # LPT bound: makespan <= 4/3 of the optimum, and >= the mean load
        assert load.max() <= (4.0 / 3.0) * max(costs.sum() / nr, costs.max()) + 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = _systems(7, seed=11)
        structs = [analysis.analyze(s) for s in systems]
        parts, _ = B.shard([B.system_flops(t) for t in structs], world)
        mine = parts[rank]
        res = {}
        for i in mine:
            x, b = M.rhs_from_xtrue(systems[i], 2, np.random.default_rng(100 + int(i)))
            _, xs = _factor_solve_np(structs[i], systems[i], b)
            res[int(i)] = (xs, x)
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        if rank == 0:
            allres = {}
            for g in gathered:
                allres.update(g)
            ok = sorted(allres) == list(range(len(systems))) and all(
                np.abs(xs - x).max() <= 1e-10 for xs, x in allres.values())
            out.put(bool(ok))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=10) is True


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_gpu_batch_matches_separate_solves(mixed):
    from pastix_b200 import gpu as G
    systems = _systems(9, seed=5) + [M.diffusion_lognormal(40, 37, 1, 0.5, np.random.default_rng(2))]
    bs = B.BatchSolver(systems, mixed=mixed, refine="cg")
    bs.solver.set_dparm(G.DPARM_EPSILON_REFINEMENT, 1e-13)
    bs.solver.numfact(bs.values())
    bl = [M.rhs_from_xtrue(s, 8, np.random.default_rng(50 + i)) for i, s in enumerate(systems)]
    b = bs.stack([t[1] for t in bl])
    x = bs.solver.solve_and_refine(b)
    for i, xs in enumerate(bs.split(x)):
        A, (xt, bi) = systems[i], bl[i]
        r = bi - A.to_scipy_full() @ xs
        assert (np.linalg.norm(r, axis=0) / np.linalg.norm(bi, axis=0)).max() <= 1e-13, i
        assert np.abs(xs - xt).max() <= 1e-9
    if not mixed:
        # FP64: the merged direct solve equals the separate ones
        xd = bs.solver.solve(b)
        for i, xs in enumerate(bs.split(xd)):
            s = G.Solver()
            s.set_iparm(G.IPARM_FACTORIZATION, G.FACT["potrf"])
            s.set_structure(bs.structs[i])
            s.set_spm(systems[i])
            s.numfact(systems[i].values)
            xi = s.solve(bl[i][1])
            assert np.abs(xs - xi).max() <= 1e-13 * np.abs(xi).max()
            s.close()
    bs.close()
