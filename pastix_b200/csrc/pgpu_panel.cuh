// Blocked panel factorization of a cblk: diagonal block factorization with
// static pivoting (kernels/core_zpotrfsp.c:68,144 core_zpotf2sp/core_zpotrfsp;
// kernels/core_zgetrfsp.c:64,138 core_zgetf2sp/core_zgetrfsp) and the panel
// TRSM of its off-diagonal rows (kernels/core_ztrsmsp.c:71), by column blocks
// of PB = 32:
//   1. one warp factorizes the PB x PB diagonal tile in shared memory;
//   2. every row below (and for LU every column to the right) is solved
//      against the tile, one thread per row;
//   3. the trailing part of the panel is updated with the solved column
//      block (a rank-PB update done as 4x4 register tiles from shared memory).
// The panel stays in global memory (L2); the tile and the solved column block
// are staged in shared memory.
#pragma once

#include "pgpu_common.cuh"

namespace pgpu {

constexpr int PB = 32;
constexpr int PBL = PB + 1;   // padded shared-memory row length

// C[i][j] -= sum_{l<K} A[i][l] * B[j][l] for i < M, j < N; when lower >= 0
// only entries with j <= i + lower are touched.  A, B in shared memory (row
// strides lda, ldb); C anywhere (row stride ldc).
template <typename T>
__device__ __forceinline__ void tile_update(T *C, int64_t ldc, const T *A, int lda, const T *B, int ldb, int M,
                                            int N, int K, int lower) {
    const int tm = (M + 3) >> 2, tn = (N + 3) >> 2;
    for (int t = threadIdx.x; t < tm * tn; t += blockDim.x) {
        const int ti = t / tn, tj = t - ti * tn;
        const int i0 = ti * 4, j0 = tj * 4;
        if (lower >= 0 && j0 > i0 + 3 + lower) continue;
        T acc[4][4];
#pragma unroll
        for (int p = 0; p < 4; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[p][q] = T(0);
        for (int l = 0; l < K; l++) {
            T a[4], b[4];
#pragma unroll
            for (int p = 0; p < 4; p++) a[p] = (i0 + p < M) ? A[(i0 + p) * lda + l] : T(0);
#pragma unroll
            for (int q = 0; q < 4; q++) b[q] = (j0 + q < N) ? B[(j0 + q) * ldb + l] : T(0);
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[p][q] += a[p] * b[q];
        }
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const int i = i0 + p;
            if (i >= M) continue;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int j = j0 + q;
                if (j >= N || (lower >= 0 && j > i + lower)) continue;
                C[(int64_t)i * ldc + j] -= acc[p][q];
            }
        }
    }
}

// Warp-synchronous factorization of the nb x nb tile (row-major, ld PBL).
// POTRF: lower Cholesky; GETRF: LU without row pivoting.  Static pivoting as
// in the reference: |a_kk| < crit -> crit (POTRF) or +-crit (GETRF).
template <typename T, bool LU>
__device__ __forceinline__ void warp_factor_tile(T *tile, int nb, T crit, int &npiv, int &nneg, int &nbad) {
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < nb; k++) {
        if (lane == 0) {
            T a = tile[k * PBL + k];
            if (!isfinite(a)) nbad++;
            if (ScalarOps<T>::absval(a) < crit) {
                a = (LU && a < T(0)) ? -crit : crit;
                npiv++;
            }
            if (!LU) {
                if (a < T(0)) nneg++;
                a = ScalarOps<T>::sqrtv(a);
            }
            tile[k * PBL + k] = a;
        }
        __syncwarp();
        const T inv = T(1) / tile[k * PBL + k];
        if (lane > k && lane < nb) tile[lane * PBL + k] *= inv;
        __syncwarp();
        if (lane > k && lane < nb) {
            const T lik = tile[lane * PBL + k];
            if (LU) {
                for (int j = k + 1; j < nb; j++) tile[lane * PBL + j] -= lik * tile[k * PBL + j];
            } else {
                for (int j = k + 1; j <= lane; j++) tile[lane * PBL + j] -= lik * tile[j * PBL + k];
            }
        }
        __syncwarp();
    }
}

// Row solves against the factorized tile (x: nb values of one row, in place).
//   POTRF rows / LU U^T rows:  x L^T = a  (L = lower of tile; unit for LU)
//   LU L rows:                 x U   = a  (U = upper of tile, non-unit)
template <typename T>
__device__ __forceinline__ void row_solve_lower_t(T *x, const T *tile, int nb, bool unit) {
    for (int j = 0; j < nb; j++) {
        T s = x[j];
        for (int l = 0; l < j; l++) s -= x[l] * tile[j * PBL + l];
        x[j] = unit ? s : s * (T(1) / tile[j * PBL + j]);
    }
}
template <typename T>
__device__ __forceinline__ void row_solve_upper(T *x, const T *tile, int nb) {
    for (int j = 0; j < nb; j++) {
        T s = x[j];
        for (int l = 0; l < j; l++) s -= x[l] * tile[l * PBL + j];
        x[j] = s * (T(1) / tile[j * PBL + j]);
    }
}

// ---------------------------------------------------------------------------
// One CTA per cblk of the level.  rows_fused(c) = h_c when h_c <= fuse_rows
// (the off-diagonal rows are solved here too), else w_c (they go to
// k_trsm_rows).  Shared memory: tile[PB][PBL] + PL[rows][PBL] (solved
// column block of L) + for LU PU[w][PBL] (solved row block of U, stored by
// column) and PO[rows][PBL] (solved column block of the U^T rows).
// ---------------------------------------------------------------------------
template <typename T, bool LU>
__global__ void __launch_bounds__(256) k_panel_factor(Meta m, const int *__restrict__ cblks, T *__restrict__ coefL,
                                                      T *__restrict__ coefU, double critd, int fuse_rows,
                                                      int pl_rows, int pu_rows, Status *st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *tile = reinterpret_cast<T *>(smem_raw);
    T *PL = tile + PB * PBL;                 // [pl_rows][PBL]: rows r1.. of the panel
    T *PU = PL + (size_t)pl_rows * PBL;      // [pu_rows][PBL]: columns r1..w (LU only)
    T *PO = PU + (size_t)pu_rows * PBL;      // [rows - w][PBL]: fused U^T rows (LU only)
    const int c = cblks[blockIdx.x];
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int rows = (h <= fuse_rows) ? h : w;
    T *A = coefL + m.coefoff[c];
    T *AU = coefU + m.coefoff[c];
    const T crit = T(critd);
    const int tid = threadIdx.x, nt = blockDim.x;
    int npiv = 0, nneg = 0, nbad = 0;
    for (int jb = 0; jb < w; jb += PB) {
        const int nb = min(PB, w - jb);
        const int r1 = jb + nb;              // first row / column after the tile
        // 1. diagonal tile
        if (tid < 32) {
            for (int e = tid; e < nb * nb; e += 32) {
                const int i = e / nb, j = e - i * nb;
                tile[i * PBL + j] = A[(int64_t)(jb + i) * ld + jb + j];
            }
            __syncwarp();
            warp_factor_tile<T, LU>(tile, nb, crit, npiv, nneg, nbad);
            for (int e = tid; e < nb * nb; e += 32) {
                const int i = e / nb, j = e - i * nb;
                if (LU || j <= i) A[(int64_t)(jb + i) * ld + jb + j] = tile[i * PBL + j];
            }
        }
        __syncthreads();
        // 2. rows below the tile (diagonal-block rows and fused off-diagonal rows)
        for (int r = r1 + tid; r < rows; r += nt) {
            T x[PB];
            T *row = A + (int64_t)r * ld + jb;
#pragma unroll
            for (int j = 0; j < PB; j++) x[j] = (j < nb) ? row[j] : T(0);
            if (LU) row_solve_upper<T>(x, tile, nb);
            else row_solve_lower_t<T>(x, tile, nb, false);
#pragma unroll
            for (int j = 0; j < PB; j++)
                if (j < nb) {
                    row[j] = x[j];
                    PL[(r - r1) * PBL + j] = x[j];
                }
        }
        if (LU) {
            // columns right of the tile inside the diagonal block: U12 = L_T^{-1} A12
            for (int col = r1 + tid; col < w; col += nt) {
                T y[PB];
#pragma unroll
                for (int i = 0; i < PB; i++) y[i] = (i < nb) ? A[(int64_t)(jb + i) * ld + col] : T(0);
                for (int i = 0; i < nb; i++) {
                    T s = y[i];
                    for (int l = 0; l < i; l++) s -= tile[i * PBL + l] * y[l];
                    y[i] = s;
                }
#pragma unroll
                for (int i = 0; i < PB; i++)
                    if (i < nb) {
                        A[(int64_t)(jb + i) * ld + col] = y[i];
                        PU[(col - r1) * PBL + i] = y[i];
                    }
            }
            // fused U^T rows: x L_T^T = a (unit)
            for (int r = w + tid; r < rows; r += nt) {
                T x[PB];
                T *row = AU + (int64_t)r * ld + jb;
#pragma unroll
                for (int j = 0; j < PB; j++) x[j] = (j < nb) ? row[j] : T(0);
                row_solve_lower_t<T>(x, tile, nb, true);
#pragma unroll
                for (int j = 0; j < PB; j++)
                    if (j < nb) {
                        row[j] = x[j];
                        PO[(r - w) * PBL + j] = x[j];
                    }
            }
        }
        __syncthreads();
        // 3. trailing update of the columns [r1, w)
        const int ncol = w - r1;
        if (ncol > 0) {
            if (LU) {
                // L rows (diagonal block + fused off-diagonal): A[r][c] -= L[r][jb:] U[jb:][c]
                tile_update<T>(A + (int64_t)r1 * ld + r1, ld, PL, PBL, PU, PBL, rows - r1, ncol, nb, -1);
                // fused U^T rows: AU[r][c] -= X[r][jb:] L[c][jb:]
                if (rows > w)
                    tile_update<T>(AU + (int64_t)w * ld + r1, ld, PO, PBL, PL, PBL, rows - w, ncol, nb, -1);
            } else {
                // diagonal block (lower triangle) and fused off-diagonal rows
                tile_update<T>(A + (int64_t)r1 * ld + r1, ld, PL, PBL, PL, PBL, w - r1, ncol, nb, 0);
                if (rows > w)
                    tile_update<T>(A + (int64_t)w * ld + r1, ld, PL + (size_t)(w - r1) * PBL, PBL, PL, PBL,
                                   rows - w, ncol, nb, -1);
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (npiv) atomicAdd(&st->nbpivots, npiv);
        if (nneg) atomicAdd(&st->negpivots, nneg);
        if (nbad) atomicAdd(&st->nonfinite, nbad);
    }
}

// ---------------------------------------------------------------------------
// Panel TRSM of the off-diagonal rows of large cblks (not fused above):
// TR rows per CTA kept in shared memory, blocked by PB columns against the
// factorized diagonal block.  chunk = {cblk, first panel row, panel select
// (0 L / 1 U), mode} with mode 0 POTRF (x L^T = a), 1 GETRF L side
// (x U = a), 2 GETRF U side (x L^T = a, unit).
// Shared memory: X[TR][w+1] + tile[PB][PBL] + P[w][PBL].
// ---------------------------------------------------------------------------
template <typename T, int TR>
__global__ void __launch_bounds__(256) k_trsm_rows(Meta m, const int4 *__restrict__ chunks, T *__restrict__ coefL,
                                                   T *__restrict__ coefU, int maxw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int4 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y, mode = ch.w;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int nrows = min(TR, h - r0);
    const int xl = maxw + 1;
    T *X = reinterpret_cast<T *>(smem_raw);                   // [TR][xl]
    T *tile = X + TR * xl;                                      // [PB][PBL]
    T *P = tile + PB * PBL;                                     // [maxw][PBL]
    const T *D = coefL + m.coefoff[c];
    T *Pan = (ch.z ? coefU : coefL) + m.coefoff[c] + (int64_t)r0 * ld;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nrows * w; e += nt) {
        const int i = e / w, j = e - i * w;
        X[i * xl + j] = Pan[(int64_t)i * ld + j];
    }
    for (int jb = 0; jb < w; jb += PB) {
        const int nb = min(PB, w - jb), r1 = jb + nb, ncol = w - r1;
        for (int e = tid; e < nb * nb; e += nt) {
            const int i = e / nb, j = e - i * nb;
            tile[i * PBL + j] = D[(int64_t)(jb + i) * ld + jb + j];
        }
        // coefficients of the trailing update, P[col - r1][l]
        for (int e = tid; e < ncol * nb; e += nt) {
            const int cc = e / nb, l = e - cc * nb;
            P[cc * PBL + l] = (mode == 1) ? D[(int64_t)(jb + l) * ld + r1 + cc]      // U[jb+l][col]
                                          : D[(int64_t)(r1 + cc) * ld + jb + l];     // L[col][jb+l]
        }
        __syncthreads();
        for (int i = tid; i < nrows; i += nt) {
            T x[PB];
#pragma unroll
            for (int j = 0; j < PB; j++) x[j] = (j < nb) ? X[i * xl + jb + j] : T(0);
            if (mode == 1) row_solve_upper<T>(x, tile, nb);
            else row_solve_lower_t<T>(x, tile, nb, mode == 2);
#pragma unroll
            for (int j = 0; j < PB; j++)
                if (j < nb) X[i * xl + jb + j] = x[j];
        }
        __syncthreads();
        if (ncol > 0) tile_update<T>(X + r1, xl, X + jb, xl, P, PBL, nrows, ncol, nb, -1);
        __syncthreads();
    }
    for (int e = tid; e < nrows * w; e += nt) {
        const int i = e / w, j = e - i * w;
        Pan[(int64_t)i * ld + j] = X[i * xl + j];
    }
}

}  // namespace pgpu
