// Blocked panel factorization of a cblk: diagonal block factorization with
// static pivoting (kernels/core_zpotrfsp.c:68,144 core_zpotf2sp/core_zpotrfsp;
// kernels/core_zgetrfsp.c:64,138 core_zgetf2sp/core_zgetrfsp;
// kernels/core_zsytrfsp.c:63,141 and kernels/core_zhetrfsp.c:63,144 for
// LDL^t / LDL^h) and the panel TRSM of its off-diagonal rows
// (kernels/core_ztrsmsp.c:71), by column blocks of PB = 32:
//   1. one warp factorizes the PB x PB diagonal tile (rows in registers);
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

// C[i][j] -= sum_{l<K} A[i][l] * op(B[j][l] s_l) for i < M, j < N (op =
// conj when CB; s_l = bscale[l] when SC, else 1); when lower >= 0 only
// entries with j <= i + lower are touched.
// A, B in shared memory (row strides lda, ldb); C anywhere (row stride ldc).
template <typename T, bool CB, bool SC = false>
__device__ __forceinline__ void tile_update(T *C, int64_t ldc, const T *A, int lda, const T *B, int ldb, int M,
                                            int N, int K, int lower, const T *bscale = nullptr) {
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
            for (int q = 0; q < 4; q++) b[q] = (j0 + q < N) ? cj<CB>(B[(j0 + q) * ldb + l]) : T(0);
            if (SC) {
                const T sl = cj<CB>(bscale[l]);
#pragma unroll
                for (int q = 0; q < 4; q++) b[q] = b[q] * sl;
            }
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[p][q] += a[p] * b[q];
        }
        // read all 16 targets before writing any: one memory latency per
        // tile instead of a read-write round trip per element (C may be in
        // global memory, where the compiler cannot reorder them itself)
        T cv[4][4];
#pragma unroll
        for (int p = 0; p < 4; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = i0 + p, j = j0 + q;
                const bool ok = i < M && j < N && !(lower >= 0 && j > i + lower);
                cv[p][q] = ok ? C[(int64_t)i * ldc + j] : T(0);
            }
#pragma unroll
        for (int p = 0; p < 4; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = i0 + p, j = j0 + q;
                if (i < M && j < N && !(lower >= 0 && j > i + lower)) C[(int64_t)i * ldc + j] = cv[p][q] - acc[p][q];
            }
    }
}

// Static pivot (sopalin: |a_kk| < crit -> crit, or -crit for a diagonal of
// negative real part in the LU / LDL forms).
template <typename T, int MODE>
__device__ __forceinline__ T static_pivot(T a, typename real_of<T>::type crit, int &npiv) {
    typedef typename real_of<T>::type R;
    if (abs_v(a) < crit) {
        npiv++;
        return T((MODE != FM_POTRF && real_v(a) < R(0)) ? -crit : crit);
    }
    return a;
}

// Warp-synchronous factorization of the nb x nb tile (row-major, ld PBL).
//   POTRF: lower Cholesky L L^h (diagonal real and positive);
//   GETRF: LU without row pivoting (unit L below, U on and above);
//   SYTRF/HETRF: unit L below, D on the diagonal (L D L^t / L D L^h).
// Lane i keeps row i of the tile in registers; the pivot, the scaled column
// and (LU) the pivot row reach the other lanes by warp shuffles, so no step
// waits on a shared-memory round trip.  The pivot is evaluated on every lane
// alike; lane 0's counters are reported.  The tile is read from and written
// back to shared memory (row-major, ld PBL).
template <typename T, int MODE>
__device__ __forceinline__ void warp_factor_tile(T *tile, int nb, typename real_of<T>::type crit, int &npiv,
                                                     int &nneg, int &nbad) {
    typedef typename real_of<T>::type R;
    constexpr bool CJ = fm_conj(MODE);
    const int lane = threadIdx.x & 31;
    T a[PB];
#pragma unroll
    for (int j = 0; j < PB; j++) a[j] = (lane < nb && j < nb) ? tile[lane * PBL + j] : T(0);
    int piv = 0, neg = 0, bad = 0;
#pragma unroll
    for (int k = 0; k < PB; k++) {
        if (k >= nb) continue;   // (not break: the loop must unroll fully to keep a[] in registers)
        T dk = shfl_v(a[k], k);
        if (!finite_v(dk)) bad++;
        dk = static_pivot<T, MODE>(dk, crit, piv);
        if (MODE == FM_POTRF) {
            if (real_v(dk) < R(0)) neg++;
            dk = sqrt_v(dk);
        }
        if (lane == k) a[k] = dk;
        const T inv = T(1) / (MODE == FM_POTRF ? cj<CJ>(dk) : dk);
        const bool below = lane > k && lane < nb;
        if (below) a[k] = a[k] * inv;
        const T lik = a[k];
        // (constant trip counts with j > k as a predicate: the nest unrolls
        // completely, so a[] stays in registers)
        if (MODE == FM_GETRF) {
#pragma unroll
            for (int j = 0; j < PB; j++) {
                if (j > k) {
                    const T ukj = shfl_v(a[j], k);
                    if (below) a[j] -= lik * ukj;
                }
            }
        } else {
            // a_ij -= l_ik op(l_jk) (Cholesky); a_ij -= l_ik d_k op(l_jk) (LDL; LDL^h takes the real part of d_k)
            const T ld = (MODE == FM_POTRF) ? lik : lik * (MODE == FM_HETRF ? T(real_v(dk)) : dk);
#pragma unroll
            for (int j = 0; j < PB; j++) {
                if (j > k) {
                    const T ljk = shfl_v(a[k], j);
                    if (below && j <= lane) a[j] -= ld * cj<CJ>(ljk);
                }
            }
            if (MODE == FM_HETRF) {
#pragma unroll
                for (int j = 0; j < PB; j++)
                    if (j > k && below && j == lane) a[j] = T(real_v(a[j]));
            }
        }
    }
    if (lane == 0) {
        npiv += piv;
        nneg += neg;
        nbad += bad;
    }
    if (lane < nb) {
#pragma unroll
        for (int j = 0; j < PB; j++)
            if (j < nb) tile[lane * PBL + j] = a[j];
    }
}

// Shared-memory form of the same factorization (the tile stays in shared
// memory, lane 0 evaluates the pivots): for kernels whose register budget
// cannot hold a row of 8-byte elements next to their other live values.
template <typename T, int MODE>
__device__ __forceinline__ void warp_factor_tile_smem(T *tile, int nb, typename real_of<T>::type crit, int &npiv,
                                                      int &nneg, int &nbad) {
    typedef typename real_of<T>::type R;
    constexpr bool CJ = fm_conj(MODE);
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < nb; k++) {
        if (lane == 0) {
            T a = tile[k * PBL + k];
            if (!finite_v(a)) nbad++;
            a = static_pivot<T, MODE>(a, crit, npiv);
            if (MODE == FM_POTRF) {
                if (real_v(a) < R(0)) nneg++;
                a = sqrt_v(a);
            }
            tile[k * PBL + k] = a;
        }
        __syncwarp();
        const T dk = tile[k * PBL + k];
        const T inv = T(1) / (MODE == FM_POTRF ? cj<CJ>(dk) : dk);
        if (lane > k && lane < nb) tile[lane * PBL + k] = tile[lane * PBL + k] * inv;
        __syncwarp();
        if (lane > k && lane < nb) {
            const T lik = tile[lane * PBL + k];
            // 8 entries per batch: their loads are issued before the stores
            // (the compiler cannot reorder shared-memory loads past stores)
            const int jend = (MODE == FM_GETRF) ? nb - 1 : lane;
            const T f = (MODE == FM_GETRF || MODE == FM_POTRF) ? lik : lik * (MODE == FM_HETRF ? T(real_v(dk)) : dk);
            for (int j0 = k + 1; j0 <= jend; j0 += 8) {
                T src[8], cur[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int j = min(j0 + u, jend);
                    src[u] = (MODE == FM_GETRF) ? tile[k * PBL + j] : cj<CJ>(tile[j * PBL + k]);
                    cur[u] = tile[lane * PBL + j];
                }
#pragma unroll
                for (int u = 0; u < 8; u++)
                    if (j0 + u <= jend) tile[lane * PBL + j0 + u] = cur[u] - f * src[u];
            }
            // LDL^h takes the real part of d_k (zher)
            if (MODE == FM_HETRF) tile[lane * PBL + lane] = T(real_v(tile[lane * PBL + lane]));
        }
        __syncwarp();
    }
}

// Row solves against the factorized tile (x: nb values of one row, in place).
//   lower_t: x op(L)^t = a, L = lower of the tile (unit when `unit`), op =
//            conj when CJ -- POTRF rows, LU U^t rows, LDL rows (unit);
//   upper:   x U = a, U = upper of the tile (non-unit) -- LU L rows.
template <typename T, bool CJ>
__device__ __forceinline__ void row_solve_lower_t(T *x, const T *tile, int nb, bool unit) {
    for (int j = 0; j < nb; j++) {
        T s = x[j];
        for (int l = 0; l < j; l++) s -= x[l] * cj<CJ>(tile[j * PBL + l]);
        x[j] = unit ? s : s * (T(1) / cj<CJ>(tile[j * PBL + j]));
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
// One CTA per job {cblk, record slot}.  rows_fused(c) = h_c when h_c <= fuse_rows
// (the off-diagonal rows are solved here too), else w_c (they go to
// k_trsm_rows).  Shared memory: tile[PB][PBL] + dinv[PB] + PL[rows][PBL]
// (solved column block) + for GETRF PU[w][PBL] (solved row block of U,
// stored by column) and PO[rows - w][PBL] (solved column block of the U^t
// rows).  For LDL, PL holds y = x D (rows times the pivots) and the trailing
// update takes its right operand as y D^{-1} = x through dinv.
// ---------------------------------------------------------------------------
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_panel_factor(Meta m, const int2 *__restrict__ jobs, T *__restrict__ coefL,
                                                      T *__restrict__ coefU, const double *critp, int fuse_rows,
                                                      int pl_rows, int pu_rows, Status *st, int64_t *prof) {
    typedef typename real_of<T>::type R;
    constexpr bool LU = (MODE == FM_GETRF);
    constexpr bool LDL = fm_ldl(MODE);
    constexpr bool CJ = fm_conj(MODE);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *tile = reinterpret_cast<T *>(smem_raw);
    T *dinv = tile + PB * PBL;               // [PB] inverse pivots (LDL)
    T *PL = dinv + PB;                       // [pl_rows][PBL]: rows r1.. of the panel
    T *PU = PL + (size_t)pl_rows * PBL;      // [pu_rows][PBL]: columns r1..w (LU only)
    T *PO = PU + (size_t)pu_rows * PBL;      // [rows - w][PBL]: fused U^T rows (LU only)
    const int2 job = jobs[blockIdx.x];
    const int c = job.x;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int rows = (h <= fuse_rows) ? h : w;
    T *A = coefL + m.coefoff[c];
    T *AU = coefU + m.coefoff[c];
    const R crit = R(*critp);
    const int tid = threadIdx.x, nt = blockDim.x;
    const uint64_t t_start = prof ? global_ns() : 0;
    int npiv = 0, nneg = 0, nbad = 0;
    for (int jb = 0; jb < w; jb += PB) {
        const int nb = min(PB, w - jb);
        const int r1 = jb + nb;              // first row / column after the tile
        // 1. diagonal tile (loaded by the whole CTA, factorized by warp 0)
        batched_copy(
            nb * nb, tid, nt, [&](int e) { const int i = e / nb, j = e - i * nb; return A[(int64_t)(jb + i) * ld + jb + j]; },
            [&](int e, T v) { const int i = e / nb, j = e - i * nb; tile[i * PBL + j] = v; });
        __syncthreads();
        if (tid < 32) {
            warp_factor_tile<T, MODE>(tile, nb, crit, npiv, nneg, nbad);
            for (int e = tid; e < nb * nb; e += 32) {
                const int i = e / nb, j = e - i * nb;
                if (LU || j <= i) A[(int64_t)(jb + i) * ld + jb + j] = tile[i * PBL + j];
            }
            if (LDL && tid < nb) dinv[tid] = T(1) / tile[tid * PBL + tid];
        }
        __syncthreads();
        // 2. rows below the tile (diagonal-block rows and fused off-diagonal rows)
        for (int r = r1 + tid; r < rows; r += nt) {
            T x[PB];
            T *row = A + (int64_t)r * ld + jb;
#pragma unroll
            for (int j = 0; j < PB; j++) x[j] = (j < nb) ? row[j] : T(0);
            if (LU) row_solve_upper<T>(x, tile, nb);
            else row_solve_lower_t<T, CJ>(x, tile, nb, LDL);
#pragma unroll
            for (int j = 0; j < PB; j++)
                if (j < nb) {
                    PL[(r - r1) * PBL + j] = x[j];            // LDL: y = x D
                    row[j] = LDL ? x[j] * dinv[j] : x[j];
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
                row_solve_lower_t<T, false>(x, tile, nb, true);
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
                tile_update<T, false>(A + (int64_t)r1 * ld + r1, ld, PL, PBL, PU, PBL, rows - r1, ncol, nb, -1);
                // fused U^T rows: AU[r][c] -= X[r][jb:] L[c][jb:]
                if (rows > w)
                    tile_update<T, false>(AU + (int64_t)w * ld + r1, ld, PO, PBL, PL, PBL, rows - w, ncol, nb, -1);
            } else {
                // diagonal block (lower triangle) and fused off-diagonal rows:
                // A[r][c] -= Y[r][jb:] op(X[c][jb:]) (Cholesky: Y = X = L;
                // LDL: Y = L D, X = Y D^{-1})
                tile_update<T, CJ, LDL>(A + (int64_t)r1 * ld + r1, ld, PL, PBL, PL, PBL, w - r1, ncol, nb, 0, dinv);
                if (rows > w)
                    tile_update<T, CJ, LDL>(A + (int64_t)w * ld + r1, ld, PL + (size_t)(w - r1) * PBL, PBL, PL, PBL,
                                            rows - w, ncol, nb, -1, dinv);
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (npiv) atomicAdd(&st->nbpivots, npiv);
        if (nneg) atomicAdd(&st->negpivots, nneg);
        if (nbad) atomicAdd(&st->nonfinite, nbad);
        if (prof) {
            prof[2 * job.y] = (int64_t)t_start;
            prof[2 * job.y + 1] = (int64_t)global_ns();
        }
    }
}

// ---------------------------------------------------------------------------
// Panel TRSM of the off-diagonal rows of large cblks (not fused above):
// TR rows per CTA kept in shared memory, blocked by PB columns against the
// factorized diagonal block.  chunk = {cblk, first panel row, panel select
// (0 L / 1 U), mode} with mode
//   0 POTRF        x op(L)^t = a          (op = conj when CJ)
//   1 GETRF L side x U = a
//   2 GETRF U side x L^t = a, unit
//   3 LDL          x D op(L)^t = a: y op(L)^t = a (unit), then x = y D^{-1}
//                  (kernels/core_zsytrfsp.c:427-460 / core_zhetrfsp.c with
//                  D op(L)^t kept in the upper triangle)
// Shared memory: X[TR][w+1] + tile[PB][PBL] + P[pch][PBL]; the trailing
// update coefficients go through P in chunks of pch columns.
// ---------------------------------------------------------------------------
template <typename T, int TR, bool CJ>
__global__ void __launch_bounds__(256) k_trsm_rows(Meta m, const int4 *__restrict__ chunks, T *__restrict__ coefL,
                                                   T *__restrict__ coefU, int maxw, int pch, int64_t *prof) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int4 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y, mode = ch.w;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int nrows = min(TR, h - r0);
    const int xl = maxw + 1;
    T *X = reinterpret_cast<T *>(smem_raw);                   // [TR][xl]
    T *tile = X + TR * xl;                                      // [PB][PBL]
    T *P = tile + PB * PBL;                                     // [pch][PBL]
    const T *D = coefL + m.coefoff[c];
    T *Pan = (ch.z ? coefU : coefL) + m.coefoff[c] + (int64_t)r0 * ld;
    const int tid = threadIdx.x, nt = blockDim.x;
    const bool cjl = CJ && mode != 2;      // conjugate the L coefficients
    const uint64_t t_start = prof ? global_ns() : 0;
    batched_copy(
        nrows * w, tid, nt, [&](int e) { const int i = e / w, j = e - i * w; return Pan[(int64_t)i * ld + j]; },
        [&](int e, T v) { const int i = e / w, j = e - i * w; X[i * xl + j] = v; });
    for (int jb = 0; jb < w; jb += PB) {
        const int nb = min(PB, w - jb), r1 = jb + nb, ncol = w - r1;
        batched_copy(
            nb * nb, tid, nt, [&](int e) { const int i = e / nb, j = e - i * nb; return D[(int64_t)(jb + i) * ld + jb + j]; },
            [&](int e, T v) { const int i = e / nb, j = e - i * nb; tile[i * PBL + j] = v; });
        __syncthreads();
        for (int i = tid; i < nrows; i += nt) {
            T x[PB];
#pragma unroll
            for (int j = 0; j < PB; j++) x[j] = (j < nb) ? X[i * xl + jb + j] : T(0);
            if (mode == 1) row_solve_upper<T>(x, tile, nb);
            else if (cjl) row_solve_lower_t<T, CJ>(x, tile, nb, mode != 0);
            else row_solve_lower_t<T, false>(x, tile, nb, mode != 0);
#pragma unroll
            for (int j = 0; j < PB; j++)
                if (j < nb) X[i * xl + jb + j] = x[j];
        }
        __syncthreads();
        for (int cc0 = 0; cc0 < ncol; cc0 += pch) {
            const int nc2 = min(pch, ncol - cc0);
            // coefficients of the trailing update, P[col - r1 - cc0][l]
            batched_copy(
                nc2 * nb, tid, nt,
                [&](int e) {
                    const int cc = e / nb, l = e - cc * nb;
                    const int col = r1 + cc0 + cc;
                    if (mode == 1) return D[(int64_t)(jb + l) * ld + col];  // U[jb+l][col]
                    const T v = D[(int64_t)col * ld + jb + l];             // L[col][jb+l]
                    return cjl ? conj_v(v) : v;
                },
                [&](int e, T v) { const int cc = e / nb, l = e - cc * nb; P[cc * PBL + l] = v; });
            __syncthreads();
            tile_update<T, false>(X + r1 + cc0, xl, X + jb, xl, P, PBL, nrows, nc2, nb, -1);
            __syncthreads();
        }
    }
    for (int e = tid; e < nrows * w; e += nt) {
        const int i = e / w, j = e - i * w;
        T v = X[i * xl + j];
        if (mode == 3) v = v * (T(1) / D[(int64_t)j * ld + j]);
        Pan[(int64_t)i * ld + j] = v;
    }
    if (prof) {
        __syncthreads();
        if (tid == 0) {
            prof[2 * blockIdx.x] = (int64_t)t_start;
            prof[2 * blockIdx.x + 1] = (int64_t)global_ns();
        }
    }
}

}  // namespace pgpu

namespace pgpu {

// ---------------------------------------------------------------------------
// Inverse of the factorized diagonal block, for the panel TRSM done as a
// GEMM (X = A_off B^t with B the inverse below, on the tensor cores for the
// single-precision factors).  B = op(L_kk)^{-1} row-major in the inverse
// workspace (inv + invoff[c], row stride ld_c), op = conj when cjp; for LDL
// (unit L) each row n is divided by d_n, so that X = A (D op(L)^t)^{-1}.
// The strict upper part of B is left untouched (zero from the allocation).
// One CTA per (cblk, 32-column block jb): columns [jb, jb+32) of the
// inverse by blocked forward substitution over the 32-row tiles below jb.
// Shared memory: X[w - jb][33] + Lb[32][kch + VK]: the rows of a 32-row tile
// left of it are staged kch columns at a time (one burst of loads per chunk),
// 16-byte aligned rows read as broadcast vectors; each tile's triangular
// solve runs on all 8 warps (lane = row, columns split across the warps).
// Launched with 256 threads.
// ---------------------------------------------------------------------------
// LU (lu != 0): job.y = jb + (kind << 20); kind 0 inverts U^t (the upper
// triangle of the diagonal block read transposed, non-unit) into the first
// slot -- B of the L-side TRSM, X = A U^{-1} -- and kind 1 the unit lower L
// into the second slot (inv_span further) -- B of the U^t-side TRSM.
// Byte offset of the L strip buffer behind X[nrow][PBL] (16-byte aligned).
__host__ __device__ inline size_t tri_inverse_lb_offset(int nrow, size_t esz) {
    return ((size_t)nrow * PBL * esz + 15) / 16 * 16;
}

// bulk_lb > 0 (the rows of L, not the U^t columns): the 32-row strip left of
// each tile and the tile itself arrive by bulk asynchronous copies, one per
// row (the rows are contiguous in the row-major panel), into two buffers of
// PB rows x bulk_lb (strip) and PB rows x (PB + VK) (tile): the copies of
// the next tile row are in flight while the current one is computed.  A
// copy that does not land within the bounded wait is counted in
// Status::timeout and the factorization reported failed.
template <typename T>
__global__ void __launch_bounds__(256) k_tri_inverse(Meta m, const int2 *__restrict__ jobs,
                                                     const T *__restrict__ coefL, T *__restrict__ inv,
                                                     int unit, int cjp, int scale_d, int lu, int kch,
                                                     T *__restrict__ ihilo, int64_t iplane, int bulk_lb,
                                                     Status *st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t tmb[2];
    __shared__ int tfail;
    const int2 jbv = jobs[blockIdx.x];
    const int c = jbv.x, jb = jbv.y & 0xFFFFF, kind = jbv.y >> 20;
    const int w = m.width[c], ld = m.ld[c];
    const int nb = min(PB, w - jb), nrow = w - jb;
    const T *D = coefL + m.coefoff[c];
    T *Inv = inv + m.invoff[c] + (kind ? inv_span(w, ld) : 0);
    const bool tr = lu && kind == 0;      // U^t: element (r, k) read at D[k][r]
    if (lu) unit = kind;
    constexpr int VK = 16 / sizeof(T) > 0 ? 16 / sizeof(T) : 1;   // k values per 16-byte load
    T *X = reinterpret_cast<T *>(smem_raw);   // [nrow][PBL]
    T *Lb = reinterpret_cast<T *>(smem_raw + tri_inverse_lb_offset(nrow, sizeof(T)));   // [PB][kch + VK]
    const int lb = kch + VK;                  // 16-byte rows
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nrow * PB; e += nt) {
        const int i = e / PB, q = e - i * PB;
        X[i * PBL + q] = (i == q && q < nb) ? T(1) : T(0);
    }
    if (bulk_lb > 0 && !tr) {
        constexpr int TLB = PB + VK;   // tile rows, 16-byte multiples
        const int slb = bulk_lb;
        auto strip = [&](int b) { return Lb + (size_t)b * (PB * (size_t)slb + PB * TLB); };
        auto tile = [&](int b) { return strip(b) + (size_t)PB * slb; };
        if (tid == 0) {
            mbar_init(smem_u32(&tmb[0]), 1);
            mbar_init(smem_u32(&tmb[1]), 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            tfail = 0;
        }
        __syncthreads();
        // thread 0: rows ib .. ib + nbi of L, columns jb .. ib (the strip) and ib .. (the tile)
        auto issue = [&](int b, int ib) {
            const int nbi = min(PB, w - ib), kn = ib - jb, tcols = (nbi + VK - 1) / VK * VK;
            const uint32_t bytes = (uint32_t)((size_t)nbi * (kn + tcols) * sizeof(T));
            mbar_arrive_expect_tx(smem_u32(&tmb[b]), bytes);
            for (int r = 0; r < nbi; r++) {
                const T *row = D + (int64_t)(ib + r) * ld;
                if (kn)
                    bulk_g2s(smem_u32(strip(b) + (size_t)r * slb), row + jb, (uint32_t)(kn * sizeof(T)),
                             smem_u32(&tmb[b]));
                bulk_g2s(smem_u32(tile(b) + (size_t)r * TLB), row + ib, (uint32_t)(tcols * sizeof(T)),
                         smem_u32(&tmb[b]));
            }
        };
        if (tid == 0) issue(0, jb);
        int stp = 0;
        for (int ib = jb; ib < w; ib += PB, stp++) {
            const int b = stp & 1, nbi = min(PB, w - ib), kn = ib - jb;
            // the other buffer was last read by the previous step (synchronized at its end)
            if (tid == 0 && ib + PB < w) issue(b ^ 1, ib + PB);
            if (!mbar_wait(smem_u32(&tmb[b]), (uint32_t)((stp >> 1) & 1))) tfail = 1;
            __syncthreads();
            if (tfail) {
                if (tid == 0) {
                    // this step's copies and, when issued, the next step's land before the CTA leaves
                    atomicAdd(&st->timeout, 1);
                    if (!mbar_wait(smem_u32(&tmb[b]), (uint32_t)((stp >> 1) & 1))) atomicAdd(&st->drain_timeout, 1);
                    if (ib + PB < w && !mbar_wait(smem_u32(&tmb[b ^ 1]), (uint32_t)(((stp + 1) >> 1) & 1)))
                        atomicAdd(&st->drain_timeout, 1);
                }
                break;
            }
            const T *Ls = strip(b), *Lt = tile(b);
            if (kn > 0) {
                // X[ib..] -= L[ib.., jb..ib) X[jb..ib): thread = rows r4..r4+3 of the strip, column q
                const int q = tid & 31, r4 = (tid >> 5) * 4;
                T acc[4] = {T(0), T(0), T(0), T(0)};
                for (int k = 0; k < kn; k += VK) {
                    T lv[4][VK];
#pragma unroll
                    for (int p = 0; p < 4; p++) {
                        const uint4 u = *reinterpret_cast<const uint4 *>(Ls + (r4 + p) * slb + k);
                        memcpy(lv[p], &u, 16);
                    }
#pragma unroll
                    for (int v = 0; v < VK; v++) {
                        const T xv = X[(k + v) * PBL + q];
#pragma unroll
                        for (int p = 0; p < 4; p++) acc[p] += (cjp ? conj_v(lv[p][v]) : lv[p][v]) * xv;
                    }
                }
                if (q < nb)
#pragma unroll
                    for (int p = 0; p < 4; p++)
                        if (r4 + p < nbi) X[(kn + r4 + p) * PBL + q] -= acc[p];
            }
            __syncthreads();
            {
                // X[ib..ib+nbi) = L_tile^{-1} X[ib..ib+nbi): warp w solves columns w, w + 8, .. (lane = row)
                const int warp = tid >> 5, lane = tid & 31;
                T y[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int q = warp + 8 * u;
                    y[u] = (lane < nbi && q < nb) ? X[(kn + lane) * PBL + q] : T(0);
                }
                T dg = lane < nbi ? Lt[lane * TLB + lane] : T(1);
                if (cjp) dg = conj_v(dg);
                const T rinv = (!unit && lane < nbi) ? T(1) / dg : T(1);
#pragma unroll
                for (int k = 0; k < PB; k++) {
                    if (k >= nbi) break;
                    T lrk = (lane > k && lane < nbi) ? Lt[lane * TLB + k] : T(0);
                    if (cjp) lrk = conj_v(lrk);
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        if (lane == k && !unit) y[u] = y[u] * rinv;
                        const T xk = shfl_v(y[u], k);
                        if (lane > k) y[u] -= lrk * xk;
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int q = warp + 8 * u;
                    if (lane < nbi && q < nb) X[(kn + lane) * PBL + q] = y[u];
                }
            }
            __syncthreads();
        }
    }
    __syncthreads();
    for (int ib = (bulk_lb > 0 && !tr) ? w : jb; ib < w; ib += PB) {
        const int nbi = min(PB, w - ib);
        // (1) X[ib..] -= L[ib.., jb..ib) X[jb..ib), kch columns of L at a time
        for (int kc0 = jb; kc0 < ib; kc0 += kch) {
            const int kn = min(kch, ib - kc0);
            if (tr)   // U^t rows are U columns: coalesce along the row index
                batched_copy(
                    nbi * kn, tid, nt,
                    [&](int e) {
                        const int k = e / nbi, r = e - k * nbi;
                        const T v = D[(int64_t)(kc0 + k) * ld + ib + r];
                        return cjp ? conj_v(v) : v;
                    },
                    [&](int e, T v) { const int k = e / nbi, r = e - k * nbi; Lb[r * lb + k] = v; });
            else
                batched_copy(
                    nbi * kn, tid, nt,
                    [&](int e) {
                        const int r = e / kn, k = e - r * kn;
                        const T v = D[(int64_t)(ib + r) * ld + kc0 + k];
                        return cjp ? conj_v(v) : v;
                    },
                    [&](int e, T v) { const int r = e / kn, k = e - r * kn; Lb[r * lb + k] = v; });
            __syncthreads();
            {
                // thread: rows r4..r4+3 of the strip, column q; the four L
                // rows come as 16-byte broadcast loads (one per row and VK k)
                const int q = tid & 31, r4 = (tid >> 5) * 4;
                T acc[4] = {T(0), T(0), T(0), T(0)};
                const T *Xc = X + (kc0 - jb) * PBL + q;
                for (int k = 0; k < kn; k += VK) {
                    T lv[4][VK];
#pragma unroll
                    for (int p = 0; p < 4; p++) {
                        const uint4 u = *reinterpret_cast<const uint4 *>(Lb + (r4 + p) * lb + k);
                        memcpy(lv[p], &u, 16);
                    }
#pragma unroll
                    for (int v = 0; v < VK; v++) {
                        const T xv = Xc[(k + v) * PBL];
#pragma unroll
                        for (int p = 0; p < 4; p++) acc[p] += lv[p][v] * xv;
                    }
                }
                if (q < nb)
#pragma unroll
                    for (int p = 0; p < 4; p++)
                        if (r4 + p < nbi) X[(ib - jb + r4 + p) * PBL + q] -= acc[p];
            }
            __syncthreads();
        }
        // (2) X[ib..ib+nbi) = L_tile^{-1} X[ib..ib+nbi), one lane per column
        batched_copy(
            nbi * nbi, tid, nt,
            [&](int e) {
                const int r = e / nbi, k = e - r * nbi;
                const T v = tr ? D[(int64_t)(ib + k) * ld + ib + r] : D[(int64_t)(ib + r) * ld + ib + k];
                return cjp ? conj_v(v) : v;
            },
            [&](int e, T v) { const int r = e / nbi, k = e - r * nbi; Lb[r * lb + k] = v; });
        __syncthreads();
        {
            // warp w solves columns w, w + 8, w + 16, w + 24 with lane = row:
            // x_k = y_k / L_kk on lane k, broadcast, y_r -= L_rk x_k below
            const int warp = tid >> 5, lane = tid & 31;
            T y[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int q = warp + 8 * u;
                y[u] = (lane < nbi && q < nb) ? X[(ib - jb + lane) * PBL + q] : T(0);
            }
            const T rinv = (!unit && lane < nbi) ? T(1) / Lb[lane * lb + lane] : T(1);
#pragma unroll
            for (int k = 0; k < PB; k++) {
                if (k >= nbi) break;
                const T lrk = (lane > k && lane < nbi) ? Lb[lane * lb + k] : T(0);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (lane == k && !unit) y[u] = y[u] * rinv;
                    const T xk = shfl_v(y[u], k);
                    if (lane > k) y[u] -= lrk * xk;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int q = warp + 8 * u;
                if (lane < nbi && q < nb) X[(ib - jb + lane) * PBL + q] = y[u];
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < nrow * nb; e += nt) {
        const int i = e / nb, q = e - i * nb;
        T v = X[i * PBL + q];
        if (scale_d) v = v * (T(1) / D[(int64_t)(jb + i) * ld + jb + i]);
        const int64_t o = (int64_t)(jb + i) * ld + jb + q;
        Inv[o] = v;
        if constexpr (std::is_same<T, float>::value) {
            if (ihilo) {   // hi / lo planes of the tensor-core operand (3xTF32)
                const int64_t io = (Inv - inv) + o;
                const float hi = tf32_round(v);
                ihilo[io] = hi;
                ihilo[iplane + io] = v - hi;
            }
        }
    }
}

// Copy the TRSM result (X of the GEMM, in the level's scratch at scroff[c],
// row stride ld_c) back into the off-diagonal rows of the panel.  One CTA per
// TRSM chunk {cblk, first row, panel, mode} of 32 rows.
// For LU the U^t rows (panel 1) come from the second half of the cblk's
// scratch (inv_span(h - w, ld) further) and go to the U coeftab.
// hilo != nullptr (single precision, TMA operands): the rows' hi / lo split
// is written too, at the coeftab offsets (U^t rows coefnbr further) of the
// planes hilo[0..plane) and hilo[plane..2 plane).
template <typename T>
__global__ void k_trsm_copyback(Meta m, const int4 *__restrict__ chunks, const int64_t *__restrict__ scroff,
                                const T *__restrict__ scr, T *__restrict__ coefL, T *__restrict__ coefU,
                                T *__restrict__ hilo, int64_t plane, int64_t coefnbr) {
    const int4 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int nr = min(32, h - r0);
    const T *src = scr + scroff[c] + (ch.z ? inv_span(h - w, ld) : 0) + (int64_t)(r0 - w) * ld;
    const int64_t doff = m.coefoff[c] + (int64_t)r0 * ld;
    T *dst = (ch.z ? coefU : coefL) + doff;
    T *hdst = hilo ? hilo + doff + (ch.z ? coefnbr : 0) : nullptr;
    batched_copy(
        nr * w, threadIdx.x, blockDim.x, [&](int e) { const int i = e / w, j = e - i * w; return src[(int64_t)i * ld + j]; },
        [&](int e, T v) {
            const int i = e / w, j = e - i * w;
            dst[(int64_t)i * ld + j] = v;
            if constexpr (std::is_same<T, float>::value) {
                if (hdst) {
                    const float hi = tf32_round(v);
                    hdst[(int64_t)i * ld + j] = hi;
                    hdst[plane + (int64_t)i * ld + j] = v - hi;
                }
            }
        });
}

}  // namespace pgpu
