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
// dst[k] >= 0: coef[dst[k]] = v; dst[k] < 0: coef[~dst[k]] = conj(v) (a
// Hermitian entry stored in the other triangle after the permutation, the
// conjugation bcsc/bcsc_zinit.c applies through __fct_conj).
template <typename T, typename Tin>
__global__ void k_fillin(int64_t nnz, const Tin *__restrict__ vals,
                         const int64_t *__restrict__ dst, T *__restrict__ coef,
                         Status *st) {
    typedef typename real_of<T>::type R;
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; k < nnz; k += stride) {
        Tin v = vals[k];
        int64_t d = dst[k];
        if (d < 0) {
            d = ~d;
            v = conj_v(v);
        }
        if (sizeof(R) == 4 && !(abs_v(v) <= 3.4028234663852886e38)) atomicAdd(&st->overflow, 1);
        coef[d] = T(v);
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
// 4 target U, 8 lower-triangle-only target (symmetric diagonal block),
// 16 scale by the pivots of c (LDL: C -= A D op(B)^t, core_zgemdm),
// 32 conjugate B (Hermitian forms: op = conj),
// 64 panel TRSM as a GEMM: X = A B^t with A the off-diagonal rows of c
//    (arow0 = w_c, M = h_c - w_c), B the inverse of its diagonal block
//    (inv + invoff[c], N = K = w_c), X stored (not accumulated) at scr + out
//    with row stride ld_c; 128: B is the cblk's second inverse (LU U^t side).
// ---------------------------------------------------------------------------
constexpr int GEMM_TM = 64, GEMM_TN = 64, GEMM_TK = 16;

struct GemmTask {
    int c, b, f, arow0, M, flags;
    int64_t out;   // flags & 64 (panel TRSM as GEMM): element offset of X in the level's scratch
};

template <typename T>
__global__ void __launch_bounds__(256) k_gemm_scatter(Meta m, const int4 *__restrict__ tiles,
                                                      const GemmTask *__restrict__ tasks,
                                                      T *__restrict__ coefL, T *__restrict__ coefU,
                                                      const T *__restrict__ inv, T *__restrict__ scr,
                                                      int64_t *prof) {
    const uint64_t t_start = prof ? global_ns() : 0;
    __shared__ T As[GEMM_TK][GEMM_TM + 4];
    __shared__ T Bs[GEMM_TK][GEMM_TN + 4];
    __shared__ T Ds[GEMM_TK];
    __shared__ int trow_s[GEMM_TM];
    const int4 tl = tiles[blockIdx.x];
    const GemmTask t = tasks[tl.x];
    const int c = t.c, b = t.b, f = t.f;
    const int K = m.width[c], ld = m.ld[c];
    const bool trsm = (t.flags & 64) != 0;
    const int N = trsm ? K : m.blrow[b] - m.bfrow[b] + 1;
    const int i0 = tl.y * GEMM_TM, j0 = tl.z * GEMM_TN;
    const T *A = ((t.flags & 1) ? coefU : coefL) + m.coefoff[c] + (int64_t)(t.arow0 + i0) * ld;
    const T *B = trsm ? inv + m.invoff[c] + ((t.flags & 128) ? inv_span(K, ld) : 0) + (int64_t)j0 * ld
                      : ((t.flags & 2) ? coefU : coefL) + m.coefoff[c] + (int64_t)(m.browoff[b] + j0) * ld;
    const int mrows = min(GEMM_TM, t.M - i0), ncols = min(GEMM_TN, N - j0);
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

    // target panel row of each tile row (binary search in f's blocks)
    if (tid < GEMM_TM && !trsm) {
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

    const bool scale_d = (t.flags & 16) != 0, conj_b = (t.flags & 32) != 0;
    const T *Dg = coefL + m.coefoff[c];
    for (int k0 = 0; k0 < K; k0 += GEMM_TK) {
        if (scale_d) {
            if (tid < GEMM_TK) Ds[tid] = (k0 + tid < K) ? Dg[(int64_t)(k0 + tid) * ld + k0 + tid] : T(0);
            __syncthreads();
        }
#pragma unroll
        for (int s = 0; s < 4; s++) {
            int e = tid + s * 256;
            int r = e >> 4, kk = e & 15;
            int kg = k0 + kk;
            T av = (r < mrows && kg < K) ? A[(int64_t)r * ld + kg] : T(0);
            T bv = (r < ncols && kg < K) ? B[(int64_t)r * ld + kg] : T(0);
            if (scale_d) av = av * Ds[kk];
            if (conj_b) bv = conj_v(bv);
            As[kk][r] = av;
            Bs[kk][r] = bv;
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

    if (trsm) {
        T *O = scr + t.out + (int64_t)i0 * ld + j0;
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const int i = ty * 4 + p;
            if (i >= mrows) continue;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int j = tx * 4 + q;
                if (j < ncols) O[(int64_t)i * ld + j] = acc[p][q];
            }
        }
        if (prof) {
            __syncthreads();
            if (tid == 0) {
                prof[2 * blockIdx.x] = (int64_t)t_start;
                prof[2 * blockIdx.x + 1] = (int64_t)global_ns();
            }
        }
        return;
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
    if (prof) {
        __syncthreads();
        if (tid == 0) {
            prof[2 * blockIdx.x] = (int64_t)t_start;
            prof[2 * blockIdx.x + 1] = (int64_t)global_ns();
        }
    }
}

// ---------------------------------------------------------------------------
// Narrow update tasks (N <= 32 rows in block b: the leaves of 2D problems and
// thin separators): one warp per 32-row slab of the task, lane i owning row
// i's N outputs in registers.  The slab's A rows and B rows are staged per
// 32-column chunk of K in the warp's shared memory (coalesced along k), then
// C[i][j] += A[i][k] op(B[j][k]) in increasing k; the same flags as
// k_gemm_scatter (U-side operands, D-scaled A for LDL, conjugated B,
// lower-triangle-only targets) and the same scatter-add into the facing cblk.
// ---------------------------------------------------------------------------
constexpr int GS_TM = 32, GS_TN = 32, GS_WARPS = 8;
template <typename T>
constexpr int gs_smem_bytes() { return GS_WARPS * 2 * 32 * 33 * (int)sizeof(T); }

template <typename T>
__global__ void __launch_bounds__(GS_WARPS * 32) k_gemm_scatter_small(Meta m, const int4 *__restrict__ tiles,
                                                                       int ntiles, const GemmTask *__restrict__ tasks,
                                                                       T *__restrict__ coefL, T *__restrict__ coefU) {
    extern __shared__ __align__(16) unsigned char gs_smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T *As = reinterpret_cast<T *>(gs_smem_raw) + warp * 2 * 32 * 33;   // [k][i], stride 33
    T *Bs = As + 32 * 33;                                               // [k][j]
    const int ti = blockIdx.x * GS_WARPS + warp;
    if (ti >= ntiles) return;                 // whole warps; only warp-level synchronization below
    const int4 tl = tiles[ti];
    const GemmTask t = tasks[tl.x];
    const int c = t.c, b = t.b, f = t.f;
    const int K = m.width[c], ld = m.ld[c];
    const int N = m.blrow[b] - m.bfrow[b] + 1;
    const int i0 = tl.y * GS_TM;
    const int mrows = min(GS_TM, t.M - i0), ncols = min(GS_TN, N);
    const T *A = ((t.flags & 1) ? coefU : coefL) + m.coefoff[c] + (int64_t)(t.arow0 + i0) * ld;
    const T *Bm = ((t.flags & 2) ? coefU : coefL) + m.coefoff[c] + (int64_t)m.browoff[b] * ld;
    const T *Dg = coefL + m.coefoff[c];
    const bool scale_d = (t.flags & 16) != 0, conj_b = (t.flags & 32) != 0;
    int tr = -1;
    if (lane < mrows) tr = panel_row_of(m, f, m.rowidx[m.rowbase[c] + t.arow0 + i0 + lane]);
    T acc[GS_TN];
#pragma unroll
    for (int j = 0; j < GS_TN; j++) acc[j] = T(0);
    for (int k0 = 0; k0 < K; k0 += 32) {
        const int kn = min(32, K - k0);
        const T dk = (scale_d && lane < kn) ? Dg[(int64_t)(k0 + lane) * ld + k0 + lane] : T(1);
        // lane = k: rows of A and B read along k (coalesced)
        for (int i = 0; i < mrows; i++) {
            T av = (lane < kn) ? A[(int64_t)i * ld + k0 + lane] : T(0);
            if (scale_d) av = av * dk;
            As[lane * 33 + i] = av;
        }
        for (int j = 0; j < ncols; j++) {
            T bv = (lane < kn) ? Bm[(int64_t)j * ld + k0 + lane] : T(0);
            if (conj_b) bv = conj_v(bv);
            Bs[lane * 33 + j] = bv;
        }
        __syncwarp();
        for (int kk = 0; kk < kn; kk++) {
            const T a = As[kk * 33 + lane];
#pragma unroll
            for (int j = 0; j < GS_TN; j++)
                if (j < ncols) acc[j] += a * Bs[kk * 33 + j];
        }
        __syncwarp();
    }
    if (tr < 0) return;
    T *C = ((t.flags & 4) ? coefU : coefL) + m.coefoff[f];
    const int ldf = m.ld[f], wf = m.width[f];
    const int tcol0 = m.bfrow[b] - m.fcol[f];
    const bool lower_only = (t.flags & 8) != 0;
#pragma unroll
    for (int j = 0; j < GS_TN; j++) {
        if (j >= ncols) break;
        const int tc = tcol0 + j;
        if (lower_only && tr < wf && tc > tr) continue;
        atomic_sub(&C[(int64_t)tr * ldf + tc], acc[j]);
    }
}

}  // namespace pgpu
