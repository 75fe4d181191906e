// Device-side construction of the bcsc equivalents from the user's CSC
// pattern (the work of bcscInit, bcsc/bcsc.c:1887, and of the coeftab fill
// map of bcsc/bcsc_zinit.c:1374 / kernels/cpucblk_zinit.c:393):
//   * per user entry k = A(i, j): its coeftab offset (the lower triangle of
//     P A P^t for symmetric / Hermitian matrices, L or U^t for general ones;
//     ~offset when a Hermitian value must be conjugated) and its Frobenius
//     weight (2 for a mirrored off-diagonal entry);
//   * the full matrix A in CSR, in the user's numbering, for the refinement's
//     SpMV (which works on vectors in that numbering, so it needs no
//     permutation around it): its entries are generated in the user's entry
//     order (entry k gives slot 2k, its symmetric mirror slot 2k + 1) and
//     stably sorted by row, so the rows list their entries in the order a
//     column-by-column pass visits them (deterministic SpMV sums).
#pragma once

#include "pgpu_common.cuh"

namespace pgpu {

struct SpmMaps {
    int n;
    int64_t nnz;
    int sym, herm;
    const int64_t *colptr, *rowptr;   // user CSC (0-based)
    const int *perm;                  // permtab: user index -> permuted
    const int *col2cblk;              // permuted column -> cblk
    int64_t coefnbr;
    int64_t *fill_dst;                // [nnz]
    int8_t *wgt;                      // [nnz]
    int *key;                         // [2 nnz] CSR row of each slot (n: no entry)
    int64_t *slot;                    // [2 nnz] slot index 2k / 2k + 1
    int *colof;                       // [nnz] user column of entry k
    int *bad;                         // set when an entry is outside the matrix or the structure
};

// one warp per user column j
__global__ void __launch_bounds__(256) k_spm_maps(Meta m, SpmMaps s) {
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= s.n) return;
    const int j = (int)gw;
    const int pj0 = s.perm[j];
    for (int64_t k = s.colptr[j] + lane; k < s.colptr[j + 1]; k += 32) {
        const int64_t i = s.rowptr[k];
        s.colof[k] = j;
        s.slot[2 * k] = 2 * k;
        s.slot[2 * k + 1] = 2 * k + 1;
        if (i < 0 || i >= s.n) {
            atomicExch(s.bad, 1);
            s.key[2 * k] = s.key[2 * k + 1] = s.n;
            s.wgt[k] = 0;
            s.fill_dst[k] = 0;
            continue;
        }
        int pi = s.perm[i], pj = pj0;
        const bool off = (i != j);
        s.wgt[k] = (s.sym && off) ? 2 : 1;
        s.key[2 * k] = (int)i;                              // the entry, in row i
        s.key[2 * k + 1] = (s.sym && off) ? j : s.n;        // its mirror, in row j
        bool flip = false;
        if (s.sym && pi < pj) {
            const int t = pi;
            pi = pj;
            pj = t;
            flip = s.herm != 0;
        }
        int64_t d = -1;
        if (pi >= pj) {
            const int c = s.col2cblk[pj];
            const int pr = panel_row_of(m, c, pi);
            if (pr >= 0) d = m.coefoff[c] + (int64_t)pr * m.ld[c] + (pj - m.fcol[c]);
        } else {   // general matrix, upper entry A(pi, pj): U^t of the cblk of column pi
            const int c = s.col2cblk[pi];
            if (s.col2cblk[pj] == c) {
                d = m.coefoff[c] + (int64_t)(pi - m.fcol[c]) * m.ld[c] + (pj - m.fcol[c]);
            } else {
                const int pr = panel_row_of(m, c, pj);
                if (pr >= 0) d = s.coefnbr + m.coefoff[c] + (int64_t)pr * m.ld[c] + (pi - m.fcol[c]);
            }
        }
        if (d < 0) {
            atomicExch(s.bad, 1);
            d = 0;
        }
        s.fill_dst[k] = flip ? ~d : d;
    }
}

// after the sort: CSR columns and value sources of the sorted slots
__global__ void k_spm_csr(int64_t fnnz, const int64_t *__restrict__ slot, const int *__restrict__ colof,
                          const int64_t *__restrict__ rowptr, int herm, int *__restrict__ ccol,
                          int64_t *__restrict__ csrc) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < fnnz; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sl = slot[q], k = sl >> 1;
        if ((sl & 1) == 0) {   // the entry itself, in row i: column j
            ccol[q] = colof[k];
            csrc[q] = k;
        } else {               // its mirror, in row j: column i (conjugated if Hermitian)
            ccol[q] = (int)rowptr[k];
            csrc[q] = herm ? ~k : k;
        }
    }
}

// CSR row pointers from the sorted row keys (first slot of each row; row n
// starts at the absent mirrors, i.e. rptr[n] is the number of entries)
__global__ void k_spm_rowptr(int n, int64_t nslots, const int *__restrict__ skey, int64_t *__restrict__ rptr) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= n; r += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = nslots;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (skey[mid] < r) lo = mid + 1; else hi = mid;
        }
        rptr[r] = lo;
    }
}

}  // namespace pgpu
