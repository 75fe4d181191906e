"""Many independent systems factorized and solved as one forest.

The configuration of 512 2D systems of uneven size is launch- and
latency-bound when each system runs alone: its elimination trees are shallow
and their leaves tiny.  Here the systems' SolverMatrix structures (each from
the reference's analysis of its own matrix) are merged into one block-diagonal
structure: the cblks of all systems sit side by side, every elimination-tree
level of every system goes into the same level launch, and one solve with the
stacked right-hand sides covers all systems.  The merge is exact -- no entry
couples two systems -- so every system's factors and solution are the ones a
separate run would produce.

Refinement runs on the merged system with the per-system stopping test of
the reference (each system until its own ||r_s||_2 / ||b_s||_2 <= eps), set
through pastix_gpu_set_segments.

Sharding over GPUs (one process per GPU): `shard()` assigns whole systems to
ranks by longest-processing-time on a per-system cost (the learned cost
model's prediction, or the flop count); there is no collective on the data
path, only a gather of per-system results.
"""
import numpy as np

from . import analysis
from . import gpu as G
from . import matrices as M


def merge_structures(structs):
    """Concatenate SolverMatrix tables (dicts of analysis.analyze) into one
    block-diagonal structure.  Returns (merged dict, column offsets)."""
    offs = np.zeros(len(structs) + 1, np.int64)
    ct, bt, br, pt, pit = [], [], [], [], []
    ocol = ocblk = oblok = obrow = 0
    for i, st in enumerate(structs):
        n = int(st["n"])
        c = np.array(st["cblktab"][:-1], np.int64, copy=True)
        c[:, 0:2] += ocol
        c[:, 2] += oblok
        c[:, 3] += obrow
        b = np.array(st["bloktab"], np.int64, copy=True)
        b[:, 0:2] += ocol
        b[:, 2:4] += ocblk
        ct.append(c)
        bt.append(b)
        br.append(np.asarray(st["browtab"], np.int64) + oblok)
        pt.append(np.asarray(st["permtab"], np.int64) + ocol)
        pit.append(np.asarray(st["peritab"], np.int64) + ocol)
        ocol += n
        ocblk += c.shape[0]
        oblok += b.shape[0]
        obrow += len(st["browtab"])
        offs[i + 1] = ocol
    sentinel = np.array([ocol, ocol, oblok, obrow], np.int64)   # {fcolnum, lcolnum, fblok, brownum} past the end
    merged = dict(n=int(ocol), cblktab=np.vstack(ct + [sentinel[None, :]]), bloktab=np.vstack(bt),
                  browtab=np.concatenate(br), permtab=np.concatenate(pt), peritab=np.concatenate(pit))
    return merged, offs


def merge_systems(systems):
    """Block-diagonal SparseSystem of `systems` (same mtxtype)."""
    colptr = [np.zeros(1, np.int64)]
    rows, vals = [], []
    ocol = onnz = 0
    for s in systems:
        colptr.append(np.asarray(s.colptr[1:], np.int64) + onnz)
        rows.append(np.asarray(s.rowptr, np.int64) + ocol)
        vals.append(s.values)
        ocol += s.n
        onnz += int(s.colptr[-1])
    return M.SparseSystem(n=int(ocol), colptr=np.concatenate(colptr), rowptr=np.concatenate(rows),
                          values=np.concatenate(vals), mtxtype=systems[0].mtxtype, grid=(int(ocol), 1, 1),
                          name="batch_%d" % len(systems), meta={})


def system_flops(struct, fact="potrf"):
    """Per-system algorithmic factorization flops (the reference's sum1d
    model, symbol/symbol_cost.c pastixSymbolGetFlops)."""
    ct, bt = struct["cblktab"], struct["bloktab"]
    w = (ct[:-1, 1] - ct[:-1, 0] + 1).astype(np.float64)
    fb = ct[:, 2]
    rows = (bt[:, 1] - bt[:, 0] + 1).astype(np.float64)
    csum = np.concatenate([[0.0], np.cumsum(rows)])
    h = csum[fb[1:]] - csum[fb[:-1]]
    m = h - w
    N = w
    if fact == "getrf":
        diag = (0.5 * N * (N * (N - N / 3.0 - 1.0) + N) + 2.0 / 3.0 * N) + (0.5 * N * (N * (N - N / 3.0) - N) + N / 6.0)
        upd = 2.0 * m * N * (N + 1) + 2.0 * m * m * N
    else:
        diag = N * ((N / 6.0 + 0.5) * N + 1.0 / 3.0) + N * ((N / 6.0) * N - 1.0 / 6.0)
        upd = m * N * (N + 1) + N * m * (m + 1)
    return float(np.sum(diag + np.where(m > 0, upd, 0.0)))


def shard(costs, nranks):
    """Longest-processing-time assignment of systems to ranks: returns a list
    of index arrays (one per rank) and the predicted per-rank load."""
    order = np.argsort(-np.asarray(costs, np.float64), kind="stable")
    load = np.zeros(nranks)
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += costs[i]
    return [np.array(sorted(p), np.int64) for p in parts], load


class BatchSolver:
    """Factorize and solve a list of independent systems as one forest."""

    def __init__(self, systems, fact="potrf", mixed=False, refine="cg", device=0, structs=None):
        self.systems = systems
        self.structs = structs if structs is not None else [analysis.analyze(s) for s in systems]
        self.struct, self.offsets = merge_structures(self.structs)
        self.merged = merge_systems(systems)
        s = G.Solver(device=device)
        s.set_iparm(G.IPARM_FACTORIZATION, G.FACT[fact])
        s.set_iparm(G.IPARM_MIXED, 1 if mixed else 0)
        s.set_iparm(G.IPARM_REFINEMENT, G.REFINE[refine])
        s.set_structure(self.struct)
        s.set_spm(self.merged)
        s.set_segments(self.offsets)
        self.solver = s

    @property
    def n(self):
        return self.merged.n

    def values(self):
        return self.merged.values

    def stack(self, blocks):
        """Per-system right-hand sides (n_s x nrhs each) -> one n x nrhs block."""
        return np.asfortranarray(np.vstack(blocks))

    def split(self, X):
        return [X[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.systems))]

    def close(self):
        self.solver.close()
