"""Learned cost model of the factorization tasks.

The reference ranks and maps its tasks with offline-fitted polynomial
kernel models (common/models.c, blend/cost.c).  Here the factorization
itself records the device time of every task (pastix_gpu_record_tasks: a
cblk's panel factorization, a TRSM row chunk, an update-GEMM tile), and a
small MLP trained on those records by the library's own CUDA kernels
(pastix_gpu_mlp_*) predicts the time of a task from its shape.  Its uses:

  * ordering inside a level launch: per-cblk predicted cost (panel + TRSM +
    GEMM tiles) handed to pastix_gpu_set_cblk_priority, costlier first;
  * sharding independent systems over GPUs (pastix_b200.batch.shard): a
    system's cost is the sum of its tasks' predictions.

Without a trained network the analytic flop count of each task stands in
(FlopModel, a per-kind log-linear fit of time on flops, or the raw flops).

Features of a task (11): one-hot kind (panel, TRSM, FMA GEMM, tensor-core
GEMM), log2 of its three sizes ((w, h, rows solved in the panel kernel),
(w, rows, w) or (K, M, N)), log2 of the element size, LU and LDL flags,
log2 of its flops.
"""
import ctypes as C

import numpy as np

from . import gpu as G

NFEAT = 11
KINDS = ("panel", "trsm", "gemm", "gemm_tc")
FORMS = {"potrf": 0, "getrf": 1, "sytrf": 2, "hetrf": 3}

# launch geometry of build_fact_plan (pastix_gpu.cu)
TRSM_TR, GEMM_TM, GEMM_TN, TC_BM, TC_BN = 32, 64, 64, 128, 128


def fuse_rows_for(lu, esz):
    if esz <= 4:
        return 256 if lu else 1024
    if esz <= 8:
        return 96 if lu else 512
    return 48 if lu else 256


def _lib():
    L = G.load()
    if not hasattr(L, "_mlp_ready"):
        P, I64, I, D = C.c_void_p, C.c_int64, C.c_int, C.c_double
        L.pastix_gpu_record_tasks.argtypes = [P, I]
        L.pastix_gpu_task_records.argtypes = [P, P, P, P]
        L.pastix_gpu_task_times.argtypes = [P, P, P]
        L.pastix_gpu_set_cblk_priority.argtypes = [P, P]
        L.pastix_gpu_mlp_init.argtypes = [C.POINTER(P), I, I, I, C.c_uint64]
        L.pastix_gpu_mlp_params.argtypes = [P, P, P]
        L.pastix_gpu_mlp_set_params.argtypes = [P, P]
        L.pastix_gpu_mlp_forward.argtypes = [P, I64, P, P]
        L.pastix_gpu_mlp_gradient.argtypes = [P, I64, P, P, P, P]
        L.pastix_gpu_mlp_train.argtypes = [P, I64, P, P, I, D, P]
        L.pastix_gpu_mlp_free.argtypes = [C.POINTER(P)]
        L.pastix_gpu_mlp_free.restype = None
        L._mlp_ready = True
    return L


# --- task records ------------------------------------------------------------
def record_tasks(solver, on=True):
    G._check("pastix_gpu_record_tasks", _lib().pastix_gpu_record_tasks(solver._h, 1 if on else 0))


def task_records(solver):
    """(info (n, 8) int64, ns (n,)) of the last numfact run with recording on."""
    L = _lib()
    cnt = np.zeros(1, np.int64)
    G._check("pastix_gpu_task_records", L.pastix_gpu_task_records(solver._h, G._p(cnt), None, None))
    n = int(cnt[0])
    info = np.zeros((n, 8), np.int64)
    ns = np.zeros(n, np.float64)
    G._check("pastix_gpu_task_records", L.pastix_gpu_task_records(solver._h, G._p(cnt), G._p(info), G._p(ns)))
    return info, ns


def task_times(solver):
    """(n, 2) int64 start/end device timestamps (ns) of the same records."""
    L = _lib()
    cnt = np.zeros(1, np.int64)
    G._check("pastix_gpu_task_times", L.pastix_gpu_task_times(solver._h, G._p(cnt), None))
    t = np.zeros((int(cnt[0]), 2), np.int64)
    G._check("pastix_gpu_task_times", L.pastix_gpu_task_times(solver._h, G._p(cnt), G._p(t)))
    return t


def set_cblk_priority(solver, prio):
    p = None if prio is None else np.ascontiguousarray(prio, np.float64)
    G._check("pastix_gpu_set_cblk_priority", _lib().pastix_gpu_set_cblk_priority(solver._h, G._p(p)))


def task_flops(info):
    kind = info[:, 0]
    a, b, c = (info[:, k].astype(np.float64) for k in (2, 3, 4))
    return np.select([kind == 0, kind == 1],
                     [a ** 3 / 3.0 + np.maximum(c - a, 0.0) * a * a, b * a * a],
                     2.0 * a * b * c)


def features(info):
    kind = info[:, 0]
    a, b, c = (info[:, k].astype(np.float64) for k in (2, 3, 4))
    X = np.zeros((info.shape[0], NFEAT))
    X[np.arange(len(kind)), kind] = 1.0
    X[:, 4] = np.log2(1.0 + a)
    X[:, 5] = np.log2(1.0 + b)
    X[:, 6] = np.log2(1.0 + np.where(kind == 1, a, c))
    X[:, 7] = np.log2(info[:, 6].astype(np.float64))
    X[:, 8] = (info[:, 7] == 1)
    X[:, 9] = (info[:, 7] >= 2)
    X[:, 10] = np.log2(1.0 + task_flops(info))
    return X


def plan_tasks(struct, fact="potrf", esz=8, use_tc=False, complex_=False):
    """The task list build_fact_plan launches for this structure (same
    records as pastix_gpu_task_records, without the timings)."""
    ct, bt = np.asarray(struct["cblktab"]), np.asarray(struct["bloktab"])
    form = FORMS[fact]
    lu = form == 1
    ldl = form >= 2
    fuse = fuse_rows_for(lu, esz)
    flags_sym = 8 | (16 if ldl else 0) | (32 if (complex_ and form in (0, 3)) else 0)
    rows_b = bt[:, 1] - bt[:, 0] + 1
    out = []
    for c in range(ct.shape[0] - 1):
        w = int(ct[c, 1] - ct[c, 0] + 1)
        b0, b1 = int(ct[c, 2]), int(ct[c + 1, 2])
        rowoff = np.concatenate([[0], np.cumsum(rows_b[b0:b1])])
        h = int(rowoff[-1])
        out.append((0, c, w, h, h if h <= fuse else w, b1 - b0))
        if h > fuse:
            for r0 in range(w, h, TRSM_TR):
                if lu:
                    out.append((1, c, w, min(32, h - r0), 1, 0))
                    out.append((1, c, w, min(32, h - r0), 2, 1))
                else:
                    out.append((1, c, w, min(32, h - r0), 3 if ldl else 0, 0))
        for b in range(b0 + 1, b1):
            N = int(rows_b[b])

            def add(arow0, flags):
                M = h - arow0
                if M <= 0:
                    return
                tc = use_tc and w >= 32 and M >= 64 and N >= 32 and M * N >= 128 * 64
                bm, bn = (TC_BM, TC_BN) if tc else (GEMM_TM, GEMM_TN)
                for tm in range(-(-M // bm)):
                    for tn in range(-(-N // bn)):
                        if (flags & 8) and tm < tn:
                            continue
                        out.append((3 if tc else 2, c, w, min(bm, M - tm * bm), min(bn, N - tn * bn), flags))

            if not lu:
                add(int(rowoff[b - b0]), flags_sym)
            else:
                add(int(rowoff[b - b0]), 2)
                if b + 1 < b1:
                    add(int(rowoff[b + 1 - b0]), 1 | 4)
    info = np.zeros((len(out), 8), np.int64)
    if out:
        info[:, :6] = np.array(out, np.int64)
    info[:, 6] = esz
    info[:, 7] = form
    return info


def cblk_costs(info, pred, cblknbr):
    """Per-cblk sum of the predicted task times."""
    return np.bincount(info[:, 1], weights=pred, minlength=cblknbr)


# --- models ------------------------------------------------------------------
class FlopModel:
    """Analytic fallback: per task kind, log(time) = a + b log(flops), least
    squares on recorded tasks; unfitted it returns the flop count itself."""

    def __init__(self):
        self.coef = {}

    def fit(self, info, ns):
        f = np.log(1.0 + task_flops(info))
        y = np.log(np.maximum(ns, 1.0))
        for k in range(len(KINDS)):
            sel = info[:, 0] == k
            if sel.sum() >= 2:
                A = np.stack([np.ones(sel.sum()), f[sel]], 1)
                self.coef[k] = np.linalg.lstsq(A, y[sel], rcond=None)[0]
        return self

    def predict(self, info):
        fl = task_flops(info)
        out = fl.copy()
        for k, (a, b) in self.coef.items():
            sel = info[:, 0] == k
            out[sel] = np.exp(a + b * np.log(1.0 + fl[sel]))
        return out


class MLPCostModel:
    """The network (trained on the GPU by pastix_gpu_mlp_train) on
    standardized features, regressing standardized log-time."""

    def __init__(self, hidden=32, seed=0, device=0):
        self.hidden = hidden
        self.h = C.c_void_p()
        G._check("pastix_gpu_mlp_init", _lib().pastix_gpu_mlp_init(C.byref(self.h), device, NFEAT, hidden, seed))
        self.mu = np.zeros(NFEAT)
        self.sd = np.ones(NFEAT)
        self.ymu, self.ysd = 0.0, 1.0
        self.trained = False

    def _x(self, info):
        return np.ascontiguousarray((features(info) - self.mu) / self.sd)

    def fit(self, info, ns, steps=3000, lr=3e-3):
        X = features(info)
        self.mu = X.mean(0)
        self.sd = np.where(X.std(0) > 0, X.std(0), 1.0)
        y = np.log(np.maximum(ns, 1.0))
        self.ymu, self.ysd = float(y.mean()), float(y.std() if y.std() > 0 else 1.0)
        Xs = self._x(info)
        ys = np.ascontiguousarray((y - self.ymu) / self.ysd)
        loss = np.zeros(1)
        G._check("pastix_gpu_mlp_train", _lib().pastix_gpu_mlp_train(self.h, Xs.shape[0], G._p(Xs), G._p(ys),
                                                                     int(steps), float(lr), G._p(loss)))
        self.trained = True
        return float(loss[0])

    def predict(self, info):
        if info.shape[0] == 0:
            return np.zeros(0)
        Xs = self._x(info)
        y = np.zeros(Xs.shape[0])
        G._check("pastix_gpu_mlp_forward", _lib().pastix_gpu_mlp_forward(self.h, Xs.shape[0], G._p(Xs), G._p(y)))
        return np.exp(y * self.ysd + self.ymu)

    def params(self):
        cnt = np.zeros(1, np.int64)
        _lib().pastix_gpu_mlp_params(self.h, None, G._p(cnt))
        p = np.zeros(int(cnt[0]))
        G._check("pastix_gpu_mlp_params", _lib().pastix_gpu_mlp_params(self.h, G._p(p), G._p(cnt)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float64)
        G._check("pastix_gpu_mlp_set_params", _lib().pastix_gpu_mlp_set_params(self.h, G._p(p)))

    def gradient(self, X, t):
        X = np.ascontiguousarray(X, np.float64)
        t = np.ascontiguousarray(t, np.float64)
        g = np.zeros(len(self.params()))
        loss = np.zeros(1)
        G._check("pastix_gpu_mlp_gradient", _lib().pastix_gpu_mlp_gradient(self.h, X.shape[0], G._p(X), G._p(t),
                                                                           G._p(g), G._p(loss)))
        return float(loss[0]), g

    def close(self):
        if self.h:
            _lib().pastix_gpu_mlp_free(C.byref(self.h))
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def log_error(pred, ns):
    """Median |log(pred / measured)| -- the prediction error reported."""
    return float(np.median(np.abs(np.log(np.maximum(pred, 1e-9)) - np.log(np.maximum(ns, 1.0)))))


def system_costs(structs, model, fact="potrf", esz=8, use_tc=False):
    """Predicted factorization cost of each system: the sum over its tasks."""
    out = []
    for st in structs:
        info = plan_tasks(st, fact, esz, use_tc)
        out.append(float(model.predict(info).sum()))
    return np.array(out)


# --- judged by measured time ---------------------------------------------------
def record_batch(systems, fact="potrf", mixed=False):
    """Task records (info, ns) of one factorization of `systems` merged into
    one forest, recording on (one task per CTA; the second of two runs)."""
    from . import batch as B
    bs = B.BatchSolver(systems, fact=fact, mixed=mixed)
    try:
        record_tasks(bs.solver)
        bs.solver.numfact(bs.values())
        bs.solver.numfact(bs.values())
        return task_records(bs.solver)
    finally:
        bs.close()


def train_models(train_systems, fact="potrf", mixed=False, hidden=32, steps=2000, seed=3):
    """The network and the flop model fitted on the same recorded tasks."""
    info, ns = record_batch(train_systems, fact, mixed)
    mlp = MLPCostModel(hidden=hidden, seed=seed)
    mlp.fit(info, ns, steps=steps, lr=3e-3)
    flop = FlopModel().fit(info, ns)
    return mlp, flop


def heldout_errors(models, test_systems, fact="potrf", mixed=False):
    """Median |log(pred / measured)| of each model on systems it was not
    trained on."""
    info, ns = record_batch(test_systems, fact, mixed)
    return [log_error(m.predict(info), ns) for m in models]


def numfact_ms_with_priority(solver, prio, values, repeats=3):
    """Median device time of the factorization with the level launches
    ordered by `prio` (per-cblk cost; None: cblk order)."""
    set_cblk_priority(solver, prio)
    solver.numfact(values)                         # plan rebuilt with the new order
    t = []
    for _ in range(repeats):
        solver.numfact(values)
        t.append(solver.stats()["numfact_ms"])
    set_cblk_priority(solver, None)
    return float(np.median(t))


def shard_makespan_ms(systems, structs, parts, fact="potrf", mixed=True, nrhs=8, repeats=2):
    """Measured per-shard time-to-solution (numfact + solve + refinement,
    device ms) of each rank's shard run on this GPU one after the other, and
    the makespan (the slowest shard): what an LPT assignment decides."""
    from . import batch as B
    from . import matrices as M
    times = []
    for p in parts:
        if len(p) == 0:
            times.append(0.0)
            continue
        bs = B.BatchSolver([systems[i] for i in p], fact=fact, mixed=mixed, structs=[structs[i] for i in p])
        try:
            rhs = [M.rhs_from_xtrue(systems[i], nrhs, np.random.default_rng(1000 + int(i)))[1] for i in p]
            b = bs.stack(rhs)
            best = []
            for _ in range(repeats + 1):
                bs.solver.numfact(bs.values())
                bs.solver.solve_and_refine(b)
                st = bs.solver.stats()
                best.append(st["numfact_ms"] + st["solve_ms"] + st["refine_ms"])
            times.append(float(np.median(best[1:])))
        finally:
            bs.close()
    return max(times), times
