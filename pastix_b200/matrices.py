"""Seeded synthetic sparse systems for the five benchmark configurations.

All matrices live on an nx*ny*nz grid whose vertex (x, y, z) has index
x + nx*(y + ny*z), the numbering the reference's grid nested dissection
(order/order_grids.c:303 `pastixOrderGrid`) assumes.  Matrices are returned in
0-based CSC; symmetric and Hermitian matrices keep only their lower triangle
(as the reference's SPM generators store them), general ones keep both.

Configurations (sizes as named by the benchmark):
  laplacian_7pt      7-point Laplacian, diagonal 6, off-diagonals -1 (20^3: n=8000)
  diffusion_lognormal 7/5-point variable-coefficient diffusion, face
                     coefficients lognormal(0, sigma) per edge, Dirichlet faces
                     (one more lognormal coefficient per boundary face added to
                     the diagonal) (100^3, sigma=1; 2D sides U{32..256}, sigma=0.5)
  convdiff_upwind    -lap(u) + Pe (1,1,1).grad(u), first-order upwind, unit
                     diffusion, h = 1/(n+1), scaled by h^2:
                     diag 6 + 3 Pe h, backward neighbours -(1 + Pe h),
                     forward neighbours -1 (80^3, Pe=10)
  magnetic_laplacian A_ij = -exp(i theta_ij) on edges (theta U[0, 2pi) per edge),
                     A_ii = 6 - sigma, Hermitian indefinite (60^3, sigma=0.5)
"""
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

# Arithmetic and symmetry codes of the reference's interface
# (include/pastix/api.h:296-302, 457-460).
PastixFloat, PastixDouble, PastixComplex32, PastixComplex64 = 2, 3, 4, 5
PastixGeneral, PastixSymmetric, PastixHermitian = 111, 112, 113


@dataclass
class SparseSystem:
    n: int
    colptr: np.ndarray          # int64 [n+1]
    rowptr: np.ndarray          # int64 [nnz]
    values: np.ndarray          # float64 or complex128 [nnz]
    mtxtype: int                # PastixGeneral / PastixSymmetric / PastixHermitian
    grid: tuple                 # (nx, ny, nz)
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def flttype(self):
        return PastixComplex64 if np.iscomplexobj(self.values) else PastixDouble

    @property
    def nnz(self):
        return int(self.colptr[-1])

    def to_scipy_full(self):
        """Full (both triangles) scipy CSC matrix."""
        A = sp.csc_matrix((self.values, self.rowptr, self.colptr), shape=(self.n, self.n))
        if self.mtxtype == PastixGeneral:
            return A
        d = sp.diags(A.diagonal())
        At = A.T.conj() if self.mtxtype == PastixHermitian else A.T
        return (A + At - d).tocsc()


def _grid_index(nx, ny, nz):
    return np.arange(nx * ny * nz, dtype=np.int64).reshape(nz, ny, nx)


def grid_edges(nx, ny, nz):
    """Edges (lo, hi, axis) of the 7-point (5-point if nz=1) grid graph,
    x-edges first, then y, then z; lo < hi always."""
    g = _grid_index(nx, ny, nz)
    out = []
    for axis, (a, b) in enumerate([(g[:, :, :-1], g[:, :, 1:]),
                                   (g[:, :-1, :], g[:, 1:, :]),
                                   (g[:-1], g[1:])]):
        if a.size:
            out.append((a.ravel(), b.ravel(), np.full(a.size, axis, np.int8)))
    lo = np.concatenate([o[0] for o in out])
    hi = np.concatenate([o[1] for o in out])
    ax = np.concatenate([o[2] for o in out])
    return lo, hi, ax


def _assemble_lower(n, diag, lo, hi, vals_lower):
    """CSC of the lower triangle: diagonal + entries (row=hi, col=lo)."""
    rows = np.concatenate([np.arange(n, dtype=np.int64), hi])
    cols = np.concatenate([np.arange(n, dtype=np.int64), lo])
    vals = np.concatenate([diag, vals_lower])
    A = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A


def _pack(A, mtxtype, grid, name, **meta):
    return SparseSystem(n=A.shape[0], colptr=A.indptr.astype(np.int64),
                        rowptr=A.indices.astype(np.int64), values=A.data.copy(),
                        mtxtype=mtxtype, grid=grid, name=name, meta=meta)


def laplacian_7pt(nx, ny=None, nz=None):
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    n = nx * ny * nz
    lo, hi, _ = grid_edges(nx, ny, nz)
    dim = 3 if nz > 1 else 2
    A = _assemble_lower(n, np.full(n, 2.0 * dim), lo, hi, np.full(lo.size, -1.0))
    return _pack(A, PastixSymmetric, (nx, ny, nz), "laplacian_%dx%dx%d" % (nx, ny, nz))


def diffusion_lognormal(nx, ny, nz, sigma, rng):
    n = nx * ny * nz
    lo, hi, _ = grid_edges(nx, ny, nz)
    c = rng.lognormal(0.0, sigma, lo.size)
    deg = np.bincount(lo, minlength=n) + np.bincount(hi, minlength=n)
    nface = (6 if nz > 1 else 4) - deg            # Dirichlet faces per cell
    nb = int(nface.sum())
    cb = rng.lognormal(0.0, sigma, nb)
    owner = np.repeat(np.arange(n), nface)
    diag = np.bincount(lo, c, n) + np.bincount(hi, c, n) + np.bincount(owner, cb, n)
    A = _assemble_lower(n, diag, lo, hi, -c)
    return _pack(A, PastixSymmetric, (nx, ny, nz),
                 "diffusion_lognormal_%dx%dx%d" % (nx, ny, nz), sigma=sigma)


def convdiff_upwind(nx, ny, nz, pe):
    n = nx * ny * nz
    h = 1.0 / (max(nx, ny, nz) + 1)
    lo, hi, _ = grid_edges(nx, ny, nz)
    dim = 3 if nz > 1 else 2
    diag = np.full(n, 2.0 * dim + dim * pe * h)
    rows = np.concatenate([np.arange(n), hi, lo])
    cols = np.concatenate([np.arange(n), lo, hi])
    # row hi sees its backward neighbour lo: upwind -(1 + Pe h); row lo sees
    # its forward neighbour hi: -1.
    vals = np.concatenate([diag, np.full(lo.size, -(1.0 + pe * h)), np.full(lo.size, -1.0)])
    A = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return _pack(A, PastixGeneral, (nx, ny, nz), "convdiff_upwind_%dx%dx%d" % (nx, ny, nz), pe=pe)


def magnetic_laplacian(nx, ny, nz, shift, rng):
    n = nx * ny * nz
    lo, hi, _ = grid_edges(nx, ny, nz)
    theta = rng.uniform(0.0, 2.0 * np.pi, lo.size)
    dim = 3 if nz > 1 else 2
    diag = np.full(n, 2.0 * dim - shift, dtype=np.complex128)
    # A[lo, hi] = -exp(i theta); lower entry A[hi, lo] is its conjugate
    A = _assemble_lower(n, diag, lo, hi, -np.exp(-1j * theta))
    return _pack(A, PastixHermitian, (nx, ny, nz), "magnetic_laplacian_%dx%dx%d" % (nx, ny, nz),
                 shift=shift)


def rhs_from_xtrue(system, nrhs, rng):
    """x_true ~ U[-1, 1] (complex: both parts), b = A x_true, column-major n x nrhs."""
    n = system.n
    if np.iscomplexobj(system.values):
        x = rng.uniform(-1, 1, (n, nrhs)) + 1j * rng.uniform(-1, 1, (n, nrhs))
    else:
        x = rng.uniform(-1, 1, (n, nrhs))
    b = system.to_scipy_full() @ x
    return np.asfortranarray(x), np.asfortranarray(b)


# --- the five benchmark configurations ------------------------------------
def config(cid, scale=1.0, seed=0):
    """Return (list of SparseSystem, dict) for configuration `cid` (1..5).

    `scale` < 1 shrinks the grid sides (used by tests); the dict names the
    factorization, refinement and RHS count the configuration uses."""
    rng = np.random.default_rng(seed)
    s = lambda k: max(3, int(round(k * scale)))
    if cid == 1:
        return [laplacian_7pt(s(20))], dict(fact="potrf", refine="cg", nrhs=1)
    if cid == 2:
        k = s(100)
        return [diffusion_lognormal(k, k, k, 1.0, rng)], dict(fact="potrf", refine="cg", nrhs=1)
    if cid == 3:
        k = s(80)
        return [convdiff_upwind(k, k, k, 10.0)], dict(fact="getrf", refine="gmres", nrhs=4)
    if cid == 4:
        nsys = max(1, int(round(512 * scale)))
        sides = rng.integers(32, 257, nsys)
        if scale < 1.0:
            sides = np.maximum(4, (sides * scale).astype(int))
        systems = [diffusion_lognormal(int(q), int(q), 1, 0.5, rng) for q in sides]
        return systems, dict(fact="potrf", refine="cg", nrhs=8)
    if cid == 5:
        k = s(60)
        return [magnetic_laplacian(k, k, k, 0.5, rng)], dict(fact="hetrf", refine="gmres", nrhs=4)
    raise ValueError(cid)
