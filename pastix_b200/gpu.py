"""ctypes front-end of libpastix_gpu.so (include/pastix_gpu.h).

`Solver` mirrors the reference's task interface (include/pastix.h:88-110):
pastixInit -> Solver(...), pastix_task_numfact -> numfact(), pastix_task_solve
-> solve(), pastix_task_refine -> refine(), with the same iparm/dparm meaning
and the same error codes (raised as PastixGpuError).  The structure produced
by the analysis (SolverMatrix arrays + ordering) is handed over once.

There is no CPU fallback: if the CUDA library is missing or no GPU is
present, the constructor raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "libpastix_gpu.so")

# include/pastix/api.h indices (same values as include/pastix_gpu.h)
IPARM_FACTORIZATION, IPARM_STATIC_PIVOTING, IPARM_REFINEMENT = 43, 45, 51
IPARM_NBITER, IPARM_ITERMAX, IPARM_GMRES_IM, IPARM_MIXED, IPARM_SIZE = 52, 53, 54, 71, 80
DPARM_EPSILON_REFINEMENT, DPARM_RELATIVE_ERROR, DPARM_EPSILON_MAGN_CTRL = 1, 2, 3
DPARM_FACT_TIME, DPARM_FACT_FLOPS, DPARM_FACT_THFLOPS = 10, 11, 12
DPARM_SOLV_TIME, DPARM_REFINE_TIME, DPARM_A_NORM, DPARM_SIZE = 17, 22, 23, 26
FACT = {"potrf": 0, "sytrf": 1, "getrf": 2, "hetrf": 4}
REFINE = {"gmres": 0, "cg": 1}
ERRORS = {1: "PASTIX_ERR_UNKNOWN", 2: "PASTIX_ERR_ALLOC", 3: "PASTIX_ERR_NOTIMPLEMENTED",
          4: "PASTIX_ERR_OUTOFMEMORY", 6: "PASTIX_ERR_INTERNAL", 7: "PASTIX_ERR_BADPARAMETER"}

EXPORTS = ["pastix_gpu_init", "pastix_gpu_structure", "pastix_gpu_spm", "pastix_gpu_numfact",
           "pastix_gpu_solve", "pastix_gpu_refine", "pastix_gpu_solve_and_refine",
           "pastix_gpu_get_params", "pastix_gpu_set_iparm", "pastix_gpu_set_dparm",
           "pastix_gpu_coeftab", "pastix_gpu_stats", "pastix_gpu_finalize"]


class PastixGpuError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__("%s returned %s (%d)" % (fn, ERRORS.get(code, "?"), code))
        self.code = code


_lib = None


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError("libpastix_gpu.so is not built: run `python -m pastix_b200.build`")
        L = C.CDLL(LIB)
        P, I64, I, D = C.c_void_p, C.c_int64, C.c_int, C.c_double
        L.pastix_gpu_init.argtypes = [C.POINTER(P), I, P, P]
        L.pastix_gpu_structure.argtypes = [P, I64, I64, P, I64, P, I64, P, P, P]
        L.pastix_gpu_spm.argtypes = [P, I, I, I64, P, P]
        L.pastix_gpu_numfact.argtypes = [P, P]
        L.pastix_gpu_solve.argtypes = [P, I64, P, I64]
        L.pastix_gpu_refine.argtypes = [P, I64, P, I64, P, I64]
        L.pastix_gpu_solve_and_refine.argtypes = [P, I64, P, I64, P, I64]
        L.pastix_gpu_get_params.argtypes = [P, P, P]
        L.pastix_gpu_set_iparm.argtypes = [P, I, I64]
        L.pastix_gpu_set_dparm.argtypes = [P, I, D]
        L.pastix_gpu_coeftab.argtypes = [P, P, P]
        L.pastix_gpu_stats.argtypes = [P, P]
        L.pastix_gpu_set_segments.argtypes = [P, I64, P]
        L.pastix_gpu_finalize.argtypes = [C.POINTER(P)]
        L.pastix_gpu_finalize.restype = None
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    if isinstance(a, int):          # raw device pointer
        return C.c_void_p(a)
    if hasattr(a, "data_ptr"):      # torch tensor
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _check(fn, rc):
    if rc != 0:
        raise PastixGpuError(fn, rc)


def init_params():
    """pastixInitParam (common/api.c:411-560) for the entries this layer reads."""
    iparm = np.zeros(IPARM_SIZE, np.int64)
    dparm = np.zeros(DPARM_SIZE, np.float64)
    iparm[IPARM_FACTORIZATION] = FACT["getrf"]
    iparm[IPARM_REFINEMENT] = REFINE["gmres"]
    iparm[IPARM_ITERMAX] = 250
    iparm[IPARM_GMRES_IM] = 25
    dparm[DPARM_EPSILON_REFINEMENT] = -1.0
    dparm[DPARM_EPSILON_MAGN_CTRL] = 0.0
    return iparm, dparm


class Solver:
    """One GPU solver instance (the device half of a pastix_data_t)."""

    def __init__(self, iparm=None, dparm=None, device=0):
        L = load()
        ip, dp = init_params()
        if iparm is not None:
            ip[:] = iparm
        if dparm is not None:
            dp[:] = dparm
        self._h = C.c_void_p()
        _check("pastix_gpu_init", L.pastix_gpu_init(C.byref(self._h), device, _p(ip), _p(dp)))
        self.n = None
        self.dtype = np.float64      # right-hand-side / solution type (complex128 for complex matrices)

    # -- parameters --------------------------------------------------------
    def set_iparm(self, idx, v):
        _check("pastix_gpu_set_iparm", load().pastix_gpu_set_iparm(self._h, idx, int(v)))

    def set_dparm(self, idx, v):
        _check("pastix_gpu_set_dparm", load().pastix_gpu_set_dparm(self._h, idx, float(v)))

    def params(self):
        ip = np.zeros(IPARM_SIZE, np.int64)
        dp = np.zeros(DPARM_SIZE, np.float64)
        _check("pastix_gpu_get_params", load().pastix_gpu_get_params(self._h, _p(ip), _p(dp)))
        return ip, dp

    def stats(self):
        s = np.zeros(16, np.float64)
        _check("pastix_gpu_stats", load().pastix_gpu_stats(self._h, _p(s)))
        keys = ["numfact_launches", "solve_launches", "refine_launches", "numfact_ms", "solve_ms",
                "refine_ms", "gemm_ms", "gemm_launches", "diag_ms", "trsm_ms", "gemm_flops", "tc_ms",
                "tc_flops", "tc_timeouts", "graph_replayed", "spm_ms"]
        return dict(zip(keys, s.tolist()))

    def phase_log(self):
        """Timeline of the last directly launched numfact: a list of
        (stream, phase, level, start_ms, end_ms); phase 0 diagonal blocks,
        1 panel TRSM, 2 FMA update GEMMs, 3 tensor-core update GEMMs."""
        L = load()
        if not hasattr(L, "_phase_log_ready"):
            L.pastix_gpu_phase_log.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
            L._phase_log_ready = True
        cnt = np.zeros(1, np.int64)
        _check("pastix_gpu_phase_log", L.pastix_gpu_phase_log(self._h, _p(cnt), None, None))
        info = np.zeros((max(int(cnt[0]), 1), 3), np.int64)
        t = np.zeros((max(int(cnt[0]), 1), 2), np.float64)
        _check("pastix_gpu_phase_log", L.pastix_gpu_phase_log(self._h, _p(cnt), _p(info), _p(t)))
        k = int(cnt[0])
        return [tuple(int(v) for v in info[i]) + (float(t[i, 0]), float(t[i, 1])) for i in range(k)]

    # -- structure / pattern -----------------------------------------------
    def set_structure(self, st):
        """st: dict with n, cblktab (cblknbr+1,4), bloktab (bloknbr,4), browtab, permtab, peritab."""
        self._st = {k: np.ascontiguousarray(st[k], np.int64)
                    for k in ("cblktab", "bloktab", "browtab", "permtab", "peritab")}
        s = self._st
        self.n = int(st["n"])
        rc = load().pastix_gpu_structure(self._h, self.n, s["cblktab"].shape[0] - 1, _p(s["cblktab"]),
                                         s["bloktab"].shape[0], _p(s["bloktab"]), s["browtab"].size,
                                         _p(s["browtab"]), _p(s["permtab"]), _p(s["peritab"]))
        _check("pastix_gpu_structure", rc)

    def set_spm(self, system):
        self._colptr = np.ascontiguousarray(system.colptr, np.int64)
        self._rowptr = np.ascontiguousarray(system.rowptr, np.int64)
        rc = load().pastix_gpu_spm(self._h, system.mtxtype, system.flttype, system.n,
                                   _p(self._colptr), _p(self._rowptr))
        _check("pastix_gpu_spm", rc)
        self.dtype = np.complex128 if np.iscomplexobj(system.values) else np.float64

    def set_segments(self, offsets):
        """Batch of independent systems: offsets[i] = first unknown of system i
        (offsets[-1] = n); refinement then applies each system's own test."""
        self._seg = np.ascontiguousarray(offsets, np.int64)
        rc = load().pastix_gpu_set_segments(self._h, len(self._seg) - 1, _p(self._seg))
        _check("pastix_gpu_set_segments", rc)

    # -- numerical tasks ---------------------------------------------------
    def numfact(self, values):
        v = values if hasattr(values, "data_ptr") or isinstance(values, int) else np.ascontiguousarray(values)
        _check("pastix_gpu_numfact", load().pastix_gpu_numfact(self._h, _p(v)))

    def solve(self, b):
        """Returns x with A x = b (b: n or n x nrhs, host numpy, Fortran order)."""
        x = np.array(b, dtype=self.dtype, order="F", copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        _check("pastix_gpu_solve", load().pastix_gpu_solve(self._h, nrhs, _p(x), self.n))
        return x

    def solve_inplace(self, B, nrhs, ldb):
        """B: host array or device pointer/tensor, overwritten with X."""
        _check("pastix_gpu_solve", load().pastix_gpu_solve(self._h, nrhs, _p(B), ldb))

    def refine(self, b, x):
        b = np.array(b, dtype=self.dtype, order="F")
        x = np.array(x, dtype=self.dtype, order="F", copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        _check("pastix_gpu_refine", load().pastix_gpu_refine(self._h, nrhs, _p(b), self.n, _p(x), self.n))
        return x

    def solve_and_refine(self, b):
        b = np.array(b, dtype=self.dtype, order="F")
        x = np.zeros_like(b, order="F")
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        rc = load().pastix_gpu_solve_and_refine(self._h, nrhs, _p(b), self.n, _p(x), self.n)
        _check("pastix_gpu_solve_and_refine", rc)
        return x

    def coeftab(self):
        """(L, U) in the reference's 1D panel layout, cblk after cblk."""
        ct = self._st["cblktab"]
        bt = self._st["bloktab"]
        nc = ct.shape[0] - 1
        total = 0
        for c in range(nc):
            w = ct[c, 1] - ct[c, 0] + 1
            b0, b1 = ct[c, 2], ct[c + 1, 2]
            h = int(np.sum(bt[b0:b1, 1] - bt[b0:b1, 0] + 1))
            total += h * w
        ip, _ = self.params()
        mixed = ip[IPARM_MIXED] != 0
        if self.dtype == np.complex128:
            dt = np.complex64 if mixed else np.complex128
        else:
            dt = np.float32 if mixed else np.float64
        Lc = np.zeros(total, dt)
        Uc = np.zeros(total, dt) if ip[IPARM_FACTORIZATION] == FACT["getrf"] else None
        _check("pastix_gpu_coeftab", load().pastix_gpu_coeftab(self._h, _p(Lc), _p(Uc)))
        return Lc, Uc

    def close(self):
        if self._h:
            load().pastix_gpu_finalize(C.byref(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
