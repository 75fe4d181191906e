// Numerical factorization kernels: coeftab fill-in, diagonal-block
// factorization with static pivoting, panel TRSM and the update GEMM with its
// indexed scatter-add into the facing column block.
#pragma once

#include "pgpu_common.cuh"

namespace pgpu {

// ---------------------------------------------------------------------------
// Fill-in (kernels/cpucblk_zinit.c:393 cpucblk_zfillin_fr and, for the mixed
// factorization, kernels/cpucblk_zcinit.c:81 cpucblk_zcfillin_fr): every
// value of the user's matrix lands at its precomputed coeftab offset.  The
// coeftab was zeroed before.  A value that does not fit the factor type
// (single precision) is flagged, as cpucblk_zccheck_overflow does.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_fillin(int64_t nnz, const double *__restrict__ vals,
                         const int64_t *__restrict__ dst, T *__restrict__ coef,
                         Status *st) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < nnz; k += stride) {
        double v = vals[k];
        if (sizeof(T) == 4 && fabs(v) > 3.4028234663852886e38) atomicAdd(&st->overflow, 1);
        coef[dst[k]] = (T)v;
    }
}

// ---------------------------------------------------------------------------
// Diagonal block factorization, one CTA per cblk of the level.
//   POTRF: kernels/core_zpotrfsp.c:68 core_zpotf2sp -- |a_kk| < crit gives
//          a_kk := crit (a static pivot); a negative pivot is reported.
//   GETRF: kernels/core_zgetrfsp.c:64 core_zgetf2sp -- |a_kk| < crit gives
//          a_kk := +-crit with the sign of a_kk; no row pivoting.
// The w x w block is factorized in shared memory when it fits, in place in
// global memory otherwise.  Column k is scaled by the reciprocal of the
// pivot, as the reference does (alpha = 1/a_kk; scal).
// ---------------------------------------------------------------------------
template <typename T, bool LU>
__global__ void k_diag_factor(Meta m, const int *__restrict__ cblks, T *__restrict__ coef,
                              double crit, int smem_cap, Status *st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *S = reinterpret_cast<T *>(smem_raw);
    __shared__ T piv_s;
    const int c = cblks[blockIdx.x];
    const int w = m.width[c];
    const int ldg = m.ld[c];
    T *G = coef + m.coefoff[c];
    // smem_cap: elements of dynamic shared memory this launch was given
    const bool in_smem = (w * w <= smem_cap);
    T *A = in_smem ? S : G;
    const int lda = in_smem ? w : ldg;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (in_smem) {
        for (int e = tid; e < w * w; e += nt) {
            int i = e / w, j = e - i * w;
            S[e] = (LU || j <= i) ? G[(int64_t)i * ldg + j] : T(0);
        }
        __syncthreads();
    }
    int npiv = 0, nneg = 0, nbad = 0;
    for (int k = 0; k < w; k++) {
        if (tid == 0) {
            T akk = A[k * lda + k];
            if (!isfinite(akk)) nbad++;
            if (ScalarOps<T>::absval(akk) < T(crit)) {
                if (LU) akk = (akk < T(0)) ? T(-crit) : T(crit);
                else akk = T(crit);
                npiv++;
            }
            if (!LU) {
                if (akk < T(0)) nneg++;
                akk = ScalarOps<T>::sqrtv(akk);
            }
            A[k * lda + k] = akk;
            piv_s = T(1) / akk;
        }
        __syncthreads();
        const T alpha = piv_s;
        for (int i = k + 1 + tid; i < w; i += nt) A[i * lda + k] *= alpha;
        __syncthreads();
        const int r = w - k - 1;
        if (LU) {
            for (int e = tid; e < r * r; e += nt) {
                int i = k + 1 + e / r, j = k + 1 + e % r;
                A[i * lda + j] -= A[i * lda + k] * A[k * lda + j];
            }
        } else {
            // lower triangle of the trailing block, rows i >= j
            for (int e = tid; e < r * r; e += nt) {
                int i = k + 1 + e / r, j = k + 1 + e % r;
                if (j <= i) A[i * lda + j] -= A[i * lda + k] * A[j * lda + k];
            }
        }
        __syncthreads();
    }
    if (in_smem) {
        for (int e = tid; e < w * w; e += nt) {
            int i = e / w, j = e - i * w;
            if (LU || j <= i) G[(int64_t)i * ldg + j] = S[e];
        }
    }
    if (tid == 0) {
        if (npiv) atomicAdd(&st->nbpivots, npiv);
        if (nneg) atomicAdd(&st->negpivots, nneg);
        if (nbad) atomicAdd(&st->nonfinite, nbad);
    }
}

// ---------------------------------------------------------------------------
// Panel TRSM (kernels/core_ztrsmsp.c:71 core_ztrsmsp_1d): every panel row
// below the diagonal block is an independent solve against the factorized
// diagonal block D (w x w, row-major).  Three forms:
//   mode 0  POTRF       X := X L^{-T}        (Right, Lower, ConjTrans, NonUnit)
//   mode 1  GETRF on L  X := X U^{-1}        (Right, Upper, NoTrans,  NonUnit)
//   mode 2  GETRF on U  X := X L^{-T}, unit  (Right, Upper, NoTrans,  Unit) on U^T
// A CTA owns TRSM_ROWS rows kept in shared memory and eliminates column by
// column; the coefficient vector of step j is staged in shared memory.
// chunks[i] = {cblk, first panel row, panel select (0 L / 1 U), mode}.
// ---------------------------------------------------------------------------
constexpr int TRSM_ROWS = 32;

template <typename T>
__global__ void k_trsm(Meta m, const int4 *__restrict__ chunks, T *__restrict__ coefL,
                       T *__restrict__ coefU) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int4 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y, mode = ch.w;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int nrows = min(TRSM_ROWS, h - r0);
    T *X = reinterpret_cast<T *>(smem_raw);            // [TRSM_ROWS][w]
    T *v = X + TRSM_ROWS * w;                            // [w] coefficients of step j
    const T *D = coefL + m.coefoff[c];                   // diagonal block lives in L
    T *P = (ch.z ? coefU : coefL) + m.coefoff[c] + (int64_t)r0 * ld;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nrows * w; e += nt) {
        int i = e / w, j = e - i * w;
        X[e] = P[(int64_t)i * ld + j];
    }
    for (int j = 0; j < w; j++) {
        // stage coefficients: v[l] for l > j, v[j] = 1/d_jj
        for (int l = j + tid; l < w; l += nt) {
            T cval;
            if (mode == 1) cval = D[j * ld + l];   // U[j][l]
            else cval = D[l * ld + j];             // L[l][j]
            v[l] = (l == j) ? (mode == 2 ? T(1) : T(1) / cval) : cval;
        }
        __syncthreads();
        if (mode != 2)
            for (int i = tid; i < nrows; i += nt) X[i * w + j] *= v[j];
        __syncthreads();
        const int r = w - j - 1;
        for (int e = tid; e < nrows * r; e += nt) {
            int i = e / r, l = j + 1 + (e - (e / r) * r);
            X[i * w + l] -= X[i * w + j] * v[l];
        }
        __syncthreads();
    }
    for (int e = tid; e < nrows * w; e += nt) {
        int i = e / w, j = e - i * w;
        P[(int64_t)i * ld + j] = X[e];
    }
}

// ---------------------------------------------------------------------------
// Update GEMM with indexed scatter-add (kernels/core_zgemmsp.c:104
// core_zgemmsp_1d1d: W = A B^T then core_zgeadd into the facing cblk).
// Task t: source cblk c, block b facing cblk f.  A = panel rows
// [arow0, arow0 + M) of c, B = the m_b rows of block b, K = w_c; C = A B^T is
// subtracted from f at (panel row of the source row in f, column
// frownum_b + j - fcolnum_f).  Different source cblks of one level may hit the
// same target entries, so the subtraction is an atomic reduction.
// One CTA computes one GEMM_TM x GEMM_TN tile with a 4x4 register block per
// thread.  tile = {task, tile_m, tile_n, 0};
// task = {c, b, f, arow0, M, flags} with flags: 1 A from U, 2 B from U,
// 4 target U, 8 lower-triangle-only target (symmetric diagonal block).
// ---------------------------------------------------------------------------
constexpr int GEMM_TM = 64, GEMM_TN = 64, GEMM_TK = 16;

struct GemmTask {
    int c, b, f, arow0, M, flags;
};

template <typename T>
__global__ void __launch_bounds__(256) k_gemm_scatter(Meta m, const int4 *__restrict__ tiles,
                                                      const GemmTask *__restrict__ tasks,
                                                      T *__restrict__ coefL, T *__restrict__ coefU) {
    __shared__ T As[GEMM_TK][GEMM_TM + 4];
    __shared__ T Bs[GEMM_TK][GEMM_TN + 4];
    __shared__ int trow_s[GEMM_TM];
    const int4 tl = tiles[blockIdx.x];
    const GemmTask t = tasks[tl.x];
    const int c = t.c, b = t.b, f = t.f;
    const int K = m.width[c], ld = m.ld[c];
    const int N = m.blrow[b] - m.bfrow[b] + 1;
    const int i0 = tl.y * GEMM_TM, j0 = tl.z * GEMM_TN;
    const T *A = ((t.flags & 1) ? coefU : coefL) + m.coefoff[c] + (int64_t)(t.arow0 + i0) * ld;
    const T *B = ((t.flags & 2) ? coefU : coefL) + m.coefoff[c] + (int64_t)(m.browoff[b] + j0) * ld;
    const int mrows = min(GEMM_TM, t.M - i0), ncols = min(GEMM_TN, N - j0);
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

    // target panel row of each tile row (binary search in f's blocks)
    if (tid < GEMM_TM) {
        int tr = -1;
        if (tid < mrows) {
            int grow = m.rowidx[m.rowbase[c] + t.arow0 + i0 + tid];
            tr = panel_row_of(m, f, grow);
        }
        trow_s[tid] = tr;
    }

    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[a][q] = T(0);

    for (int k0 = 0; k0 < K; k0 += GEMM_TK) {
#pragma unroll
        for (int s = 0; s < 4; s++) {
            int e = tid + s * 256;
            int r = e >> 4, kk = e & 15;
            int kg = k0 + kk;
            As[kk][r] = (r < mrows && kg < K) ? A[(int64_t)r * ld + kg] : T(0);
            Bs[kk][r] = (r < ncols && kg < K) ? B[(int64_t)r * ld + kg] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GEMM_TK; kk++) {
            T a[4], bv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                a[q] = As[kk][ty * 4 + q];
                bv[q] = Bs[kk][tx * 4 + q];
            }
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[p][q] += a[p] * bv[q];
        }
        __syncthreads();
    }

    T *C = ((t.flags & 4) ? coefU : coefL) + m.coefoff[f];
    const int ldf = m.ld[f];
    const int tcol0 = m.bfrow[b] + j0 - m.fcol[f];
    const bool lower_only = (t.flags & 8) != 0;
    const int wf = m.width[f];
#pragma unroll
    for (int p = 0; p < 4; p++) {
        int i = ty * 4 + p;
        if (i >= mrows) continue;
        int tr = trow_s[i];
        if (tr < 0) continue;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int j = tx * 4 + q;
            if (j >= ncols) continue;
            int tc = tcol0 + j;
            if (lower_only && tr < wf && tc > tr) continue;
            atomic_sub(&C[(int64_t)tr * ldf + tc], acc[p][q]);
        }
    }
}

}  // namespace pgpu
