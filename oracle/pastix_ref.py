"""ctypes front-end to the PaStiX reference built by oracle/refbuild/build_ref.py.

TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and bench.py's CPU
baseline leg use this to run the reference's own CPU path (static scheduler,
sequential OpenBLAS) and to read back what it computed.  Nothing in the
shipped package imports it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libpastix_ref.so")
# the same build with the one-increment fix of core_zhetf2sp (see
# oracle/refbuild/build_ref.py HEFIX): pins the LDL^h of complex matrices
LIB_HEFIX = os.path.join(HERE, "_ref", "libpastix_ref_hefix.so")
# the same reference sources with the GPU layer plugged into its sopalinFacto,
# solve and refinement tables (pastix_b200/refplug/pastix_gpu_plug.c): not an
# oracle, the drop-in under test
LIB_GPUPLUG = os.path.join(HERE, "_ref", "libpastix_gpuplug.so")
LIBS = {None: LIB, "hefix": LIB_HEFIX, "gpuplug": LIB_GPUPLUG}

# include/pastix/api.h enumerations (iparm / dparm indices, values)
IPARM = {k: i for i, k in enumerate("""VERBOSE IO_STRATEGY NNZEROS NNZEROS_BLOCK_LOCAL ALLOCATED_TERMS
PRODUCE_STATS TRACE MC64 ORDERING ORDERING_DEFAULT SCOTCH_MT SCOTCH_SWITCH_LEVEL SCOTCH_CMIN
SCOTCH_CMAX SCOTCH_FRAT METIS_CTYPE METIS_RTYPE METIS_NO2HOP METIS_NSEPS METIS_NITER
METIS_UFACTOR METIS_COMPRESS METIS_CCORDER METIS_PFACTOR METIS_SEED METIS_DBGLVL
AMALGAMATION_LVLBLAS AMALGAMATION_LVLCBLK REORDERING_SPLIT REORDERING_STOP SPLITTING_STRATEGY
SPLITTING_LEVELS_PROJECTIONS SPLITTING_LEVELS_KWAY SPLITTING_PROJECTIONS_DEPTH
SPLITTING_PROJECTIONS_DISTANCE SPLITTING_PROJECTIONS_WIDTH MIN_BLOCKSIZE MAX_BLOCKSIZE
TASKS2D_LEVEL TASKS2D_WIDTH ALLCAND INCOMPLETE LEVEL_OF_FILL FACTORIZATION FACTO_LOOK_SIDE
STATIC_PIVOTING FREE_CSCUSER SCHUR_FACT_MODE TRANSPOSE_SOLVE SCHUR_SOLV_MODE APPLYPERM_WS
REFINEMENT NBITER ITERMAX GMRES_IM SCHEDULER THREAD_NBR SOCKET_NBR AUTOSPLIT_COMM GPU_NBR
GPU_MEMORY_PERCENTAGE GPU_MEMORY_BLOCK_SIZE GLOBAL_ALLOCATION COMPRESS_MIN_WIDTH
COMPRESS_MIN_HEIGHT COMPRESS_WHEN COMPRESS_METHOD COMPRESS_ORTHO COMPRESS_RELTOL
COMPRESS_PRESELECT COMPRESS_ILUK MIXED FTZ MPI_THREAD_LEVEL MODIFY_PARAMETER START_TASK
END_TASK FLOAT MTX_TYPE DOF_NBR SIZE""".split())}
DPARM = {k: i for i, k in enumerate("""FILL_IN EPSILON_REFINEMENT RELATIVE_ERROR EPSILON_MAGN_CTRL
ORDER_TIME SYMBFACT_TIME REORDER_TIME BLEND_TIME ANALYZE_TIME PRED_FACT_TIME FACT_TIME
FACT_FLOPS FACT_THFLOPS FACT_RLFLOPS FACT_ENERGY MEM_FR MEM_LR SOLV_TIME SOLV_FLOPS
SOLV_THFLOPS SOLV_RLFLOPS SOLV_ENERGY REFINE_TIME A_NORM COMPRESS_TOLERANCE
COMPRESS_MIN_RATIO SIZE""".split())}
FACT = {"potrf": 0, "sytrf": 1, "getrf": 2, "pxtrf": 3, "hetrf": 4}
REFINE = {"gmres": 0, "cg": 1, "sr": 2, "bicgstab": 3}
SCHED_STATIC = 1

NC, NB = 10, 8     # columns of the exported cblk / blok tables (ref_glue.c)

_libs = {}


def available(variant=None):
    return os.path.exists(LIBS[variant])


def lib(variant=None):
    if variant not in _libs:
        if not available(variant):
            raise RuntimeError("reference oracle not built: run oracle/refbuild/build_ref.py")
        L = C.CDLL(LIBS[variant])
        P, I64, I = C.c_void_p, C.c_int64, C.c_int
        L.ref_create.restype = P
        L.ref_create.argtypes = [I, I]
        L.ref_set_iparm.argtypes = [P, I, I64]
        L.ref_set_dparm.argtypes = [P, I, C.c_double]
        L.ref_get_iparm.argtypes = [P, I]
        L.ref_get_iparm.restype = I64
        L.ref_get_dparm.argtypes = [P, I]
        L.ref_get_dparm.restype = C.c_double
        L.ref_init.argtypes = [P]
        L.ref_set_matrix.argtypes = [P, I, I, I64, P, P, P]
        L.ref_analyze_grid.argtypes = [P, I64, I64, I64]
        L.ref_numfact.argtypes = [P]
        L.ref_solve.argtypes = [P, I64, P, I64]
        L.ref_refine.argtypes = [P, I64, P, I64, P, I64]
        L.ref_struct_sizes.argtypes = [P, P]
        L.ref_struct_dump.argtypes = [P, P, P, P, P, P]
        L.ref_order_cblknbr.argtypes = [P]
        L.ref_order_cblknbr.restype = I64
        L.ref_order_dump.argtypes = [P, P, P]
        L.ref_coeftab_dump.argtypes = [P, P, P]
        L.ref_destroy.argtypes = [P]
        L.ref_save_structure.argtypes = [P, C.c_char_p, C.c_char_p]
        _libs[variant] = L
    return _libs[variant]


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class RefSolver:
    """One reference pastix instance (pastix_data_t) on one matrix."""

    def __init__(self, system, fact="potrf", nthreads=1, mixed=False, refine=None,
                 eps_refine=None, itermax=None, gmres_im=None, verbose=0, iparm=None, dparm=None,
                 variant=None):
        self.variant = variant
        L = lib(variant)
        self.sys = system
        self.h = L.ref_create(nthreads, verbose)
        self.set_iparm("FACTORIZATION", FACT[fact])
        self.set_iparm("SCHEDULER", SCHED_STATIC)
        self.set_iparm("MIXED", 1 if mixed else 0)
        if refine is not None:
            self.set_iparm("REFINEMENT", REFINE[refine])
        if eps_refine is not None:
            self.set_dparm("EPSILON_REFINEMENT", eps_refine)
        if itermax is not None:
            self.set_iparm("ITERMAX", itermax)
        if gmres_im is not None:
            self.set_iparm("GMRES_IM", gmres_im)
        for k, v in (iparm or {}).items():
            self.set_iparm(k, v)
        for k, v in (dparm or {}).items():
            self.set_dparm(k, v)
        if L.ref_init(self.h):
            raise RuntimeError("pastixInit failed")
        self._keep = [np.ascontiguousarray(system.colptr, np.int64),
                      np.ascontiguousarray(system.rowptr, np.int64),
                      np.ascontiguousarray(system.values)]
        rc = L.ref_set_matrix(self.h, system.mtxtype, system.flttype, system.n,
                              *[_ptr(a) for a in self._keep])
        if rc:
            raise RuntimeError("ref_set_matrix failed")

    def set_iparm(self, k, v):
        lib(self.variant).ref_set_iparm(self.h, IPARM[k], int(v))

    def set_dparm(self, k, v):
        lib(self.variant).ref_set_dparm(self.h, DPARM[k], float(v))

    def iparm(self, k):
        return lib(self.variant).ref_get_iparm(self.h, IPARM[k])

    def dparm(self, k):
        return lib(self.variant).ref_get_dparm(self.h, DPARM[k])

    def analyze(self):
        nx, ny, nz = self.sys.grid
        rc = lib(self.variant).ref_analyze_grid(self.h, nx, ny, nz)
        if rc:
            raise RuntimeError("analysis failed: %d" % rc)

    def numfact(self):
        rc = lib(self.variant).ref_numfact(self.h)
        if rc:
            raise RuntimeError("numfact failed: %d" % rc)

    def solve(self, b):
        x = np.asfortranarray(b.copy())
        nrhs = x.shape[1] if x.ndim == 2 else 1
        rc = lib(self.variant).ref_solve(self.h, nrhs, _ptr(x), self.sys.n)
        if rc:
            raise RuntimeError("solve failed: %d" % rc)
        return x

    def refine(self, b, x):
        b = np.asfortranarray(b.copy())
        x = np.asfortranarray(x.copy())
        nrhs = x.shape[1] if x.ndim == 2 else 1
        rc = lib(self.variant).ref_refine(self.h, nrhs, _ptr(b), self.sys.n, _ptr(x), self.sys.n)
        if rc:
            raise RuntimeError("refine failed: %d" % rc)
        return x

    def structure(self):
        """The SolverMatrix and ordering, as integer tables (ref_glue.c)."""
        L = lib(self.variant)
        sz = np.zeros(16, np.int64)
        if L.ref_struct_sizes(self.h, _ptr(sz)):
            raise RuntimeError("no solver matrix")
        cblknbr, bloknbr, brownbr = int(sz[0]), int(sz[1]), int(sz[2])
        cblk = np.zeros((cblknbr + 1, NC), np.int64)
        blok = np.zeros((bloknbr + 1, NB), np.int64)
        brow = np.zeros(max(brownbr, 1), np.int64)
        perm = np.zeros(self.sys.n, np.int64)
        invp = np.zeros(self.sys.n, np.int64)
        L.ref_struct_dump(self.h, _ptr(cblk), _ptr(blok), _ptr(brow), _ptr(perm), _ptr(invp))
        oc = L.ref_order_cblknbr(self.h)
        rang = np.zeros(oc + 1, np.int64)
        tree = np.zeros(oc, np.int64)
        L.ref_order_dump(self.h, _ptr(rang), _ptr(tree))
        keys = ["cblknbr", "bloknbr", "brownbr", "coefnbr", "nodenbr", "gemmmax", "offdmax",
                "blokmax", "colmax", "factotype", "flttype", "nb2dcblk", "cblkmin2d", "cblkmax1d"]
        d = {k: int(sz[i]) for i, k in enumerate(keys)}
        d.update(cblk=cblk, blok=blok, browtab=brow[:brownbr], perm=perm, invp=invp,
                 rangtab=rang, treetab=tree)
        return d

    def coeftab(self, structure=None):
        """(L, U) factor panels, cblk after cblk, as the reference stores them."""
        st = structure or self.structure()
        cblk = st["cblk"][:-1]
        size = int(np.sum(cblk[:, 3] * (cblk[:, 1] - cblk[:, 0] + 1)))
        dt = {2: np.float32, 3: np.float64, 4: np.complex64, 5: np.complex128}[st["flttype"]]
        Lc = np.zeros(size, dt)
        Uc = np.zeros(size, dt) if st["factotype"] == FACT["getrf"] else None
        lib(self.variant).ref_coeftab_dump(self.h, _ptr(Lc), _ptr(Uc))
        return Lc, Uc

    def save_structure(self, solver_path, order_path):
        """The reference's solverSave into solver_path, the ordering in its
        ordering_save format into order_path (ref_glue.c)."""
        rc = lib(self.variant).ref_save_structure(self.h, str(solver_path).encode(), str(order_path).encode())
        if rc:
            raise RuntimeError("save_structure failed: %d" % rc)

    def close(self):
        if self.h:
            lib(self.variant).ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
