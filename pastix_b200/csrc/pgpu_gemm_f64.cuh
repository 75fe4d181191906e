// FP64 update GEMM with indexed scatter-add on the FP64 tensor cores (DMMA,
// mma.sync.aligned.m8n8k4.row.col.f64): C = A B^T of one task tile,
// subtracted from the facing cblk (kernels/core_zgemmsp.c:104
// core_zgemmsp_1d1d), or, for the panel TRSM done as a GEMM (flags & 64),
// X = A_off inv^T stored into the level's scratch.
//
// Tile 128 x 64, K staged 16 doubles at a time through a 3-stage cp.async
// ring (A and B rows padded to 20 doubles: 16-byte aligned, a fragment load
// of 8 rows x 4 doubles is the minimal two shared-memory wavefronts).  Eight
// warps as 4 (M) x 2 (N), warp tile 32 x 32 = 4 x 4 DMMA tiles of 8 x 8: per
// k-step of 4 a thread loads 4 A and 4 B doubles and issues 16 DMMAs.
// Fragments (PTX m8n8k4 .f64): A[row = lane/4][k = lane%4],
// B[k = lane%4][col = lane/4], D[row = lane/4][col = 2 (lane%4) + {0, 1}].
// The LDL^t form (flags & 16) scales A's k-th column by D_kk as it is read.
// Target rows come from the plan's row map (k_task_rowmap): one load per row.
#pragma once

#include "pgpu_common.cuh"
#include "pgpu_factor.cuh"

namespace pgpu {

constexpr int DG_BM = 128, DG_BN = 64, DG_BK = 16, DG_THREADS = 256, DG_STAGES = 3;
constexpr int DG_PITCH = DG_BK + 4;
constexpr int dg_smem_bytes() { return DG_STAGES * ((DG_BM + DG_BN) * DG_PITCH + DG_BK) * 8; }

__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(DG_THREADS, 2)
    k_gemm_scatter_dmma(Meta m, const int4 *__restrict__ tiles, const GemmTask *__restrict__ tasks,
                        double *__restrict__ coefL, double *__restrict__ coefU, const double *__restrict__ inv,
                        double *__restrict__ scr, const int *__restrict__ tmap, const int64_t *__restrict__ taux) {
    extern __shared__ __align__(16) double dg_smem[];
    double *As = dg_smem;                                   // [S][BM][PITCH]
    double *Bs = As + DG_STAGES * DG_BM * DG_PITCH;         // [S][BN][PITCH]
    double *Ds = Bs + DG_STAGES * DG_BN * DG_PITCH;         // [S][BK]
    const int4 tl = tiles[blockIdx.x];
    const GemmTask t = tasks[tl.x];
    const int c = t.c, b = t.b, f = t.f;
    const int K = m.width[c], ld = m.ld[c];
    const bool trsm = (t.flags & 64) != 0, scale_d = (t.flags & 16) != 0;
    const int N = trsm ? K : m.blrow[b] - m.bfrow[b] + 1;
    const int i0 = tl.y * DG_BM, j0 = tl.z * DG_BN;
    const double *A = ((t.flags & 1) ? coefU : coefL) + m.coefoff[c] + (int64_t)(t.arow0 + i0) * ld;
    const double *B = trsm ? inv + m.invoff[c] + ((t.flags & 128) ? inv_span(K, ld) : 0) + (int64_t)j0 * ld
                           : ((t.flags & 2) ? coefU : coefL) + m.coefoff[c] + (int64_t)(m.browoff[b] + j0) * ld;
    const double *Dg = coefL + m.coefoff[c];
    const int mrows = min(DG_BM, t.M - i0), ncols = min(DG_BN, N - j0);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp & 3, wn = warp >> 2;
    const int nk = (K + DG_BK - 1) / DG_BK;

    // target row of each of this thread's output rows (one row-map load each)
    int trow[4][2];
    {
        const int64_t tb = trsm ? 0 : taux[3 * (int64_t)tl.x];
#pragma unroll
        for (int mi = 0; mi < 4; mi++) {
            const int r = wm * 32 + mi * 8 + (lane >> 2);
            trow[mi][0] = (!trsm && r < mrows) ? tmap[tb + i0 + r] : -1;
        }
    }

    // k-block kb into stage s: 16-byte chunks, rows past the tile zero-filled
    // (columns past K read the panel's zero padding: ld >= K, rows 16-byte aligned)
    auto load = [&](int s, int kb) {
        const int k0 = kb * DG_BK;
        double *as = As + s * DG_BM * DG_PITCH, *bs = Bs + s * DG_BN * DG_PITCH;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int e = tid + q * DG_THREADS, r = e >> 3, kc = k0 + 2 * (e & 7);
            const bool v = r < mrows && kc < K;
            cp_async16(smem_u32(as + r * DG_PITCH + 2 * (e & 7)), v ? (const void *)(A + (int64_t)r * ld + kc)
                                                                    : (const void *)A, v);
        }
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int e = tid + q * DG_THREADS, r = e >> 3, kc = k0 + 2 * (e & 7);
            const bool v = r < ncols && kc < K;
            cp_async16(smem_u32(bs + r * DG_PITCH + 2 * (e & 7)), v ? (const void *)(B + (int64_t)r * ld + kc)
                                                                    : (const void *)B, v);
        }
        if (scale_d && tid < DG_BK) {
            const int k = k0 + tid;
            Ds[s * DG_BK + tid] = k < K ? Dg[(int64_t)k * ld + k] : 0.0;
        }
    };

    double acc[4][4][2];
#pragma unroll
    for (int mi = 0; mi < 4; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;

#pragma unroll
    for (int s = 0; s < DG_STAGES - 1; s++) {
        if (s < nk) load(s, s);
        cp_async_commit();
    }
    for (int kb = 0; kb < nk; kb++) {
        cp_async_wait<DG_STAGES - 2>();
        __syncthreads();   // stage kb landed; stage kb - 1 is free for the load below
        if (kb + DG_STAGES - 1 < nk) load((kb + DG_STAGES - 1) % DG_STAGES, kb + DG_STAGES - 1);
        cp_async_commit();
        const int s = kb % DG_STAGES;
        const double *as = As + s * DG_BM * DG_PITCH + (wm * 32 + (lane >> 2)) * DG_PITCH + (lane & 3);
        const double *bs = Bs + s * DG_BN * DG_PITCH + (wn * 32 + (lane >> 2)) * DG_PITCH + (lane & 3);
#pragma unroll
        for (int k4 = 0; k4 < DG_BK; k4 += 4) {
            double a[4], bv[4];
            const double dk = scale_d ? Ds[s * DG_BK + k4 + (lane & 3)] : 1.0;
#pragma unroll
            for (int mi = 0; mi < 4; mi++) a[mi] = as[mi * 8 * DG_PITCH + k4] * dk;
#pragma unroll
            for (int ni = 0; ni < 4; ni++) bv[ni] = bs[ni * 8 * DG_PITCH + k4];
#pragma unroll
            for (int mi = 0; mi < 4; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++) dmma_m8n8k4(acc[mi][ni], a[mi], bv[ni]);
        }
    }
    cp_async_wait<0>();

    if (trsm) {
        double *O = scr + t.out + (int64_t)i0 * ld + j0;
#pragma unroll
        for (int mi = 0; mi < 4; mi++) {
            const int r = wm * 32 + mi * 8 + (lane >> 2);
            if (r >= mrows) continue;
#pragma unroll
            for (int ni = 0; ni < 4; ni++)
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int j = wn * 32 + ni * 8 + 2 * (lane & 3) + e;
                    if (j < ncols) O[(int64_t)r * ld + j] = acc[mi][ni][e];
                }
        }
        return;
    }
    double *C = ((t.flags & 4) ? coefU : coefL) + m.coefoff[f];
    const int ldf = m.ld[f], wf = m.width[f];
    const int tcol0 = m.bfrow[b] + j0 - m.fcol[f];
    const bool lower_only = (t.flags & 8) != 0;
#pragma unroll
    for (int mi = 0; mi < 4; mi++) {
        const int t2 = trow[mi][0];
        if (t2 < 0) continue;
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int j = wn * 32 + ni * 8 + 2 * (lane & 3) + e;
                const int tc = tcol0 + j;
                if (j >= ncols || (lower_only && t2 < wf && tc > t2)) continue;
                atomicAdd(&C[(int64_t)t2 * ldf + tc], -acc[mi][ni][e]);
            }
    }
}

}  // namespace pgpu
