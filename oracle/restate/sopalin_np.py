"""CPU restatement (numpy) of the reference's supernodal numerical
factorization and solve, on the reference's 1D panel layout.

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path; nothing in the
shipped package imports it.  Pinned against the reference itself (the
PaStiX CPU path built by oracle/refbuild) by tests/test_oracle.py and against
the committed fixtures under tests/golden/.

Layout (kernels/cpucblk_zinit.c:220 cpucblk_zalloc_fr for a 1D cblk): cblk
after cblk, a column-major panel of `stride` rows and `width` columns; the
diagonal block is rows [0, width), off-diagonal block b follows at the row
offset given by the blocks before it.

Algorithms followed (real or complex data; the Hermitian forms POTRF = LL^h
and HETRF = LDL^h conjugate the transposed operand):
  fill-in      kernels/cpucblk_zinit.c:393  cpucblk_zfillin_fr
  POTRF        kernels/core_zpotrfsp.c:68,144,334 (core_zpotf2sp, static pivot)
  GETRF        kernels/core_zgetrfsp.c:64,217,355 (core_zgetf2sp, geadd/getmo)
  SYTRF/HETRF  kernels/core_zsytrfsp.c:63,141,482 and core_zhetrfsp.c:63,144,491
               (unit L, D on the diagonal; off-diagonal rows X (D op(L)^t) = A;
               update C -= A D op(B)^t, core_zgemdm); for HETRF the
               mathematically intended conjugation of core_zhetf2sp (the
               reference's kernels/core_zhetrfsp.c:92 passes increment 1 where
               the row has stride lda -- see oracle/refbuild/build_ref.py)
  TRSM         kernels/core_ztrsmsp.c:71  core_ztrsmsp_1d
  update GEMM  kernels/core_zgemmsp.c:104 core_zgemmsp_1d1d (GEMM + scatter-add)
  solve        kernels/solve_ztrsmsp.c:301,450 forward / backward
  CG           refinement/z_refine_grad.c:49
"""
import numpy as np
from scipy.linalg import solve_triangular


class Layout:
    """Per-cblk geometry from the SolverMatrix tables (0-based)."""

    def __init__(self, cblktab, bloktab):
        cblktab = np.asarray(cblktab)
        bloktab = np.asarray(bloktab)
        self.cblknbr = cblktab.shape[0] - 1
        self.fcol = cblktab[:-1, 0].astype(np.int64)
        self.lcol = cblktab[:-1, 1].astype(np.int64)
        self.fblok = cblktab[:, 2].astype(np.int64)
        self.frow = bloktab[:, 0].astype(np.int64)
        self.lrow = bloktab[:, 1].astype(np.int64)
        self.fcblk = bloktab[:, 3].astype(np.int64)
        self.width = self.lcol - self.fcol + 1
        m = self.lrow - self.frow + 1
        self.rowoff = np.zeros(len(m), np.int64)
        self.height = np.zeros(self.cblknbr, np.int64)
        for c in range(self.cblknbr):
            b0, b1 = self.fblok[c], self.fblok[c + 1]
            self.rowoff[b0:b1] = np.concatenate([[0], np.cumsum(m[b0:b1])[:-1]])
            self.height[c] = m[b0:b1].sum()
        self.off = np.concatenate([[0], np.cumsum(self.height * self.width)])
        self.n = int(self.lcol[-1] + 1)
        self.col2cblk = np.repeat(np.arange(self.cblknbr), self.width)

    def panel(self, arr, c):
        """Column-major view (height x width) of cblk c in a flat coeftab."""
        h, w = int(self.height[c]), int(self.width[c])
        return arr[self.off[c]:self.off[c] + h * w].reshape(w, h).T

    def rows(self, c):
        b0, b1 = self.fblok[c], self.fblok[c + 1]
        return np.concatenate([np.arange(self.frow[b], self.lrow[b] + 1) for b in range(b0, b1)])

    def panel_rows_in(self, f, grows):
        """Panel rows of cblk f holding global rows `grows` (is_block_inside_fblock)."""
        b0, b1 = self.fblok[f], self.fblok[f + 1]
        k = np.searchsorted(self.frow[b0:b1], grows, side="right") - 1 + b0
        assert np.all(grows <= self.lrow[k]), "row not in facing cblk"
        return self.rowoff[k] + grows - self.frow[k]


def ref2d_to_1d(layout, coef_ref, cblk_ref, blok_ref):
    """Convert a reference coeftab dump (1D or 2D cblks, blend/solver.h:48-54
    CBLK_LAYOUT_2D) to the 1D layout."""
    out = np.zeros(layout.off[-1], coef_ref.dtype)
    off_ref = 0
    for c in range(layout.cblknbr):
        h, w = int(layout.height[c]), int(layout.width[c])
        src = coef_ref[off_ref:off_ref + h * w]
        dst = layout.panel(out, c)
        if cblk_ref[c, 7] & 2:      # CBLK_LAYOUT_2D: blocks contiguous, ld = m_b
            for b in range(layout.fblok[c], layout.fblok[c + 1]):
                mb = int(layout.lrow[b] - layout.frow[b] + 1)
                ci = int(blok_ref[b, 4])
                dst[layout.rowoff[b]:layout.rowoff[b] + mb, :] = src[ci:ci + mb * w].reshape(w, mb).T
        else:
            dst[:, :] = src.reshape(w, h).T
        off_ref += h * w
    return out


def fillin(layout, system, perm, lu=False):
    """Scatter the (permuted) matrix into zeroed L (and U^T) coeftabs."""
    A = system.to_scipy_full().tocoo()
    pi, pj, v = perm[A.row], perm[A.col], A.data
    L = np.zeros(layout.off[-1], v.dtype)
    U = np.zeros(layout.off[-1], v.dtype) if lu else None
    low = pi >= pj
    for (ii, jj, vv, dest) in ((pi[low], pj[low], v[low], L),) + \
            (((pj[~low], pi[~low], v[~low], U),) if lu else ()):
        c = layout.col2cblk[jj]
        for cc in np.unique(c):
            sel = c == cc
            P = layout.panel(dest, cc)
            r = layout.panel_rows_in(cc, ii[sel])
            P[r, jj[sel] - layout.fcol[cc]] = vv[sel]
    return L, U


def _potf2(A, crit):
    """core_zpotf2sp on a square block (in place), returns #static pivots."""
    n = A.shape[0]
    piv = 0
    for k in range(n):
        if abs(A[k, k]) < crit:
            A[k, k] = crit
            piv += 1
        A[k, k] = np.sqrt(A[k, k].real)
        alpha = 1.0 / A[k, k]
        A[k + 1:, k] *= alpha
        A[k + 1:, k + 1:] -= np.tril(np.outer(A[k + 1:, k], np.conj(A[k + 1:, k])))
    return piv


def _getf2(A, crit):
    """core_zgetf2sp on a square block (in place), returns #static pivots."""
    n = A.shape[0]
    piv = 0
    for k in range(n):
        if abs(A[k, k]) < crit:
            A[k, k] = -crit if A[k, k].real < 0 else crit
            piv += 1
        alpha = 1.0 / A[k, k]
        A[k + 1:, k] *= alpha
        A[k + 1:, k + 1:] -= np.outer(A[k + 1:, k], A[k, k + 1:])
    return piv


def _ldlf2(A, crit, herm):
    """core_zsytf2sp / core_zhetf2sp on the lower triangle of a square block
    (in place): unit L below the diagonal, D on it.  Returns #static pivots."""
    n = A.shape[0]
    piv = 0
    for k in range(n):
        if abs(A[k, k]) < crit:
            A[k, k] = -crit if A[k, k].real < 0 else crit
            piv += 1
        d = A[k, k]
        l = A[k + 1:, k] / d
        A[k + 1:, k] = l
        if herm:
            A[k + 1:, k + 1:] -= np.tril(np.outer(l, np.conj(l))) * d.real       # zher, real alpha
            i = np.arange(k + 1, n)
            A[i, i] = A[i, i].real
        else:
            A[k + 1:, k + 1:] -= np.tril(np.outer(l * d, l))
    return piv


def _cj(herm):
    return np.conj if herm else (lambda v: v)


def factorize(layout, L, U, fact, crit):
    """Right-looking supernodal factorization in cblk order (in place).
    Returns the number of static pivots."""
    nbpiv = 0
    lu = fact == "getrf"
    ldl = fact in ("sytrf", "hetrf")
    herm = fact in ("potrf", "hetrf")
    cj = _cj(herm)
    for c in range(layout.cblknbr):
        P = layout.panel(L, c)
        w = int(layout.width[c])
        D = P[:w, :]
        if lu:
            PU = layout.panel(U, c)
            D += PU[:w, :].T                       # core_zgeadd(Trans, U -> L)
            nbpiv += _getf2(D, crit)
            PU[:w, :] = D.T                        # core_zgetmo
            if P.shape[0] > w:
                P[w:, :] = solve_triangular(np.triu(D), P[w:, :].T, trans="T", lower=False).T
                Lu = np.tril(D, -1) + np.eye(w)
                PU[w:, :] = solve_triangular(Lu, PU[w:, :].T, lower=True, unit_diagonal=True).T
        elif ldl:
            Dl = np.tril(D)
            nbpiv += _ldlf2(Dl, crit, fact == "hetrf")
            D[:, :] = Dl + np.triu(D, 1)
            if P.shape[0] > w:
                Lu = np.tril(D, -1) + np.eye(w)
                # X (D op(L)^t) = A  ->  Y op(L)^t = A, X = Y D^{-1}
                Y = cj(solve_triangular(Lu, cj(P[w:, :]).T, lower=True, unit_diagonal=True).T)
                P[w:, :] = Y / np.diag(D)[None, :]
        else:
            Dl = np.tril(D)
            nbpiv += _potf2(Dl, crit)
            D[:, :] = np.tril(Dl) + np.triu(D, 1)
            if P.shape[0] > w:
                # X op(L)^t = A  ->  L conj(X)^t = conj(A)^t for LL^h
                P[w:, :] = cj(solve_triangular(np.tril(D), cj(P[w:, :]).T, lower=True).T)
        dg = np.diag(D).copy() if ldl else None
        rows = layout.rows(c)
        b0, b1 = layout.fblok[c], layout.fblok[c + 1]
        for b in range(b0 + 1, b1):
            f = int(layout.fcblk[b])
            r0 = int(layout.rowoff[b])
            mb = int(layout.lrow[b] - layout.frow[b] + 1)
            cols = np.arange(layout.frow[b], layout.lrow[b] + 1) - layout.fcol[f]
            tr = layout.panel_rows_in(f, rows[r0:])
            F = layout.panel(L, f)
            if lu:
                PU = layout.panel(U, c)
                F[np.ix_(tr, cols)] -= P[r0:, :] @ PU[r0:r0 + mb, :].T
                if b + 1 < b1:
                    FU = layout.panel(U, f)
                    FU[np.ix_(tr[mb:], cols)] -= PU[r0 + mb:, :] @ P[r0:r0 + mb, :].T
            elif ldl:
                F[np.ix_(tr, cols)] -= (P[r0:, :] * dg[None, :]) @ cj(P[r0:r0 + mb, :]).T
            else:
                F[np.ix_(tr, cols)] -= P[r0:, :] @ cj(P[r0:r0 + mb, :]).T
    return nbpiv


def solve(layout, L, U, fact, b):
    """Forward/backward supernodal solve in the permuted numbering
    (sopalin/sequential_ztrsm.c; LDL: the diagonal solve of
    sopalin/sequential_zdiag.c between the two passes)."""
    x = np.array(b, dtype=np.result_type(L.dtype, b.dtype), copy=True)
    lu = fact == "getrf"
    ldl = fact in ("sytrf", "hetrf")
    herm = fact in ("potrf", "hetrf")
    cj = _cj(herm)
    for c in range(layout.cblknbr):
        P = layout.panel(L, c)
        w, fc = int(layout.width[c]), int(layout.fcol[c])
        D = P[:w, :]
        x[fc:fc + w] = solve_triangular(np.tril(D), x[fc:fc + w], lower=True, unit_diagonal=lu or ldl)
        if P.shape[0] > w:
            rows = layout.rows(c)[w:]
            np.subtract.at(x, rows, P[w:, :] @ x[fc:fc + w])
    if ldl:
        for c in range(layout.cblknbr):
            P = layout.panel(L, c)
            w, fc = int(layout.width[c]), int(layout.fcol[c])
            x[fc:fc + w] /= np.diag(P[:w, :])
    for c in range(layout.cblknbr - 1, -1, -1):
        P = layout.panel(L, c)
        Q = layout.panel(U, c) if lu else P
        w, fc = int(layout.width[c]), int(layout.fcol[c])
        if P.shape[0] > w:
            rows = layout.rows(c)[w:]
            x[fc:fc + w] -= (Q[w:, :].T if lu else cj(Q[w:, :]).T) @ x[rows]
        D = P[:w, :]
        if lu:
            x[fc:fc + w] = solve_triangular(np.triu(D), x[fc:fc + w], lower=False)
        else:
            x[fc:fc + w] = solve_triangular(np.tril(D), x[fc:fc + w], lower=True, trans="C" if herm else "T",
                                            unit_diagonal=ldl)
    return x
