"""Host analysis (ordering, symbolic factorization, blend split) of a grid
matrix, through libpastix_gpu.so's pastix_gpu_analyze_grid().

`analyze(system)` returns the dict pastix_b200.gpu.Solver.set_structure()
takes: n, cblktab, bloktab, browtab, permtab, peritab (+ rangtab/treetab of
the ordering).  It is pure host code (no GPU needed).
"""
import ctypes as C

import numpy as np

from . import gpu as G


def _lib():
    L = G.load()
    if not hasattr(L, "_analysis_ready"):
        P, I64 = C.c_void_p, C.c_int64
        L.pastix_gpu_analyze_grid.argtypes = [C.POINTER(P), I64, I64, I64, I64, P, P, P]
        L.pastix_gpu_analysis_sizes.argtypes = [P, P]
        L.pastix_gpu_analysis_export.argtypes = [P, P, P, P, P, P, P, P]
        L.pastix_gpu_analysis_load.argtypes = [C.POINTER(P), C.c_char_p, C.c_char_p]
        L.pastix_gpu_analysis_free.argtypes = [C.POINTER(P)]
        L.pastix_gpu_analysis_free.restype = None
        L._analysis_ready = True
    return L


def analyze(system, iparm=None):
    """Analysis of `system` (a pastix_b200.matrices.SparseSystem on a grid)."""
    L = _lib()
    nx, ny, nz = system.grid
    colptr = np.ascontiguousarray(system.colptr, np.int64)
    rowptr = np.ascontiguousarray(system.rowptr, np.int64)
    ip = None
    if iparm is not None:
        ip = np.ascontiguousarray(iparm, np.int64)
    else:
        ip = np.zeros(G.IPARM_SIZE, np.int64)
        ip[36], ip[37], ip[38], ip[39] = 160, 320, -1, 160      # common/api.c:488-491
        ip[28], ip[29] = 0, np.iinfo(np.int64).max               # reordering split/stop
    h = C.c_void_p()
    rc = L.pastix_gpu_analyze_grid(C.byref(h), nx, ny, nz, system.n, G._p(colptr), G._p(rowptr), G._p(ip))
    G._check("pastix_gpu_analyze_grid", rc)
    return _export(L, h)


def load(solver_file, order_file):
    """The structure of a saved analysis: the reference's solverSave file and
    its ordering file (pastixOrderSave), read by pastix_gpu_analysis_load;
    same dict as analyze()."""
    L = _lib()
    h = C.c_void_p()
    rc = L.pastix_gpu_analysis_load(C.byref(h), str(solver_file).encode(), str(order_file).encode())
    G._check("pastix_gpu_analysis_load", rc)
    return _export(L, h)


def _export(L, h):
    try:
        sz = np.zeros(5, np.int64)
        L.pastix_gpu_analysis_sizes(h, G._p(sz))
        n, cblknbr, bloknbr, brownbr, ocblk = (int(v) for v in sz)
        cblktab = np.zeros((cblknbr + 1, 4), np.int64)
        bloktab = np.zeros((bloknbr, 4), np.int64)
        browtab = np.zeros(max(brownbr, 1), np.int64)
        permtab = np.zeros(n, np.int64)
        peritab = np.zeros(n, np.int64)
        rangtab = np.zeros(ocblk + 1, np.int64)
        treetab = np.zeros(ocblk, np.int64)
        rc = L.pastix_gpu_analysis_export(h, G._p(cblktab), G._p(bloktab), G._p(browtab), G._p(permtab),
                                          G._p(peritab), G._p(rangtab), G._p(treetab))
        G._check("pastix_gpu_analysis_export", rc)
    finally:
        L.pastix_gpu_analysis_free(C.byref(h))
    return dict(n=n, cblktab=cblktab, bloktab=bloktab, browtab=browtab[:brownbr], permtab=permtab,
                peritab=peritab, rangtab=rangtab, treetab=treetab)
