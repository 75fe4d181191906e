// Update GEMM on the tensor cores with operands brought in by TMA
// (cp.async.bulk.tensor) instead of producer warps: the same task, tile and
// epilogue as k_gemm_scatter_tc_persistent, C = A B^T scatter-added into the
// facing cblk (kernels/core_zgemmsp.c:104 core_zgemmsp_1d1d).
//
// Operands: for 3xTF32 (SPLIT) the finished panel rows are split once into
// hi = tf32(x) and lo = x - hi by the level's split / copy-back kernels, into
// a mirror of the coeftab laid out [2][ncoef] (hi, then lo), and the
// diagonal-block inverses alike.  One tensor map per (cblk, operand kind)
// covers the panel as a 3-D tensor {K = w_c, rows = h_c, 2} with row stride
// ld_c and the hi/lo stride ncoef, so one box {32, 128, 2} lands the hi tile
// and the lo tile of a k-block (2 x 16 KB, SWIZZLE_128B, the canonical
// K-major layout the MMA descriptors expect).  Without the split the maps
// cover the coeftab itself, {K, rows, 1}.  Rows and columns past the panel
// are zero-filled by the TMA unit.
//
// Roles (192 threads, one CTA per SM walking the level's tiles):
//   warps 0-3: epilogue (TMEM -> registers -> shared transpose -> 16-byte
//              vector reductions into the target), as the persistent kernel;
//   warp 4, lane 0: TMA producer -- per k-block waits for a free stage,
//              announces the stage's bytes on its mbarrier and issues the A
//              and B box loads;
//   warp 5, lane 0: MMA issuer (tcgen05.mma into one of two TMEM
//              accumulators, commits to the stage / accumulator barriers).
// Every wait is bounded; after a time-out the producer waits (bounded) for
// the loads it issued and TMEM is freed after all roles met.  The tensor
// maps name only this GPU's memory and the loads carry no multicast.
#pragma once

#include <cuda.h>

#include "pgpu_common.cuh"
#include "pgpu_factor.cuh"
#include "pgpu_gemm_tc.cuh"

namespace pgpu {

constexpr int TMA_THREADS = 192;
constexpr int TMA_PROD_WARP = 4, TMA_MMA_WARP = 5;
// operand maps per cblk: L panel, U panel (LU), first / second diagonal-block inverse
enum { TMAP_L = 0, TMAP_U = 1, TMAP_I = 2, TMAP_I2 = 3, TMAP_KINDS = 4 };

// A stage holds two A tiles (a pair of 128-row tiles of one task sharing the
// B tile) and the B tile; hi and lo planes each for 3xTF32.
template <bool SPLIT> struct TmaCfg;
template <> struct TmaCfg<false> { static constexpr int STAGES = 4, TILES = 3, PL = 1; };
template <> struct TmaCfg<true> { static constexpr int STAGES = 2, TILES = 6, PL = 2; };
constexpr int TMA_TMEM_COLS = 512;   // two accumulator buffers x (two 128-column halves)
template <bool SPLIT>
constexpr int tma_smem_bytes() {
    return TmaCfg<SPLIT>::STAGES * TmaCfg<SPLIT>::TILES * TC_TILE_BYTES + TCP_EPI_BYTES + 1024;
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t addr, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes) : "memory");
}

// 3-D tiled TMA load into this CTA's shared memory, completing on mbar.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(mbar)
        : "memory");
}

template <bool SPLIT>
__global__ void __launch_bounds__(TMA_THREADS, 1)
    k_gemm_scatter_tc_tma(Meta m, const int4 *__restrict__ tiles, int ntiles, const GemmTask *__restrict__ tasks,
                          float *__restrict__ coefL, float *__restrict__ coefU, Status *st, float *__restrict__ scr,
                          const CUtensorMap *__restrict__ maps, const int *__restrict__ mapidx) {
    constexpr int S = TmaCfg<SPLIT>::STAGES, NT = TmaCfg<SPLIT>::TILES, PL = TmaCfg<SPLIT>::PL;
    constexpr uint32_t BOX_BYTES = (uint32_t)PL * TC_TILE_BYTES;   // one operand box (hi [+ lo])
    constexpr int QA1 = PL, QB = 2 * PL;                            // tile slots of A1 and B in a stage
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t full[S], empty[S], accf[2], acce[2], drained;
    __shared__ uint32_t tmem_base_s;
    __shared__ int fail_s;
    __shared__ int trow_s[2][TC_BM];

    const uint32_t raw = smem_u32(tc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char *sbase = tc_smem_raw + (base - raw);
    float *epi = reinterpret_cast<float *>(sbase + S * NT * TC_TILE_BYTES);   // [4][32][33]

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == TMA_MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(TMA_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&accf[b]), 1);
            mbar_init(smem_u32(&acce[b]), 4);
        }
        mbar_init(smem_u32(&drained), 1);
        fail_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;
    auto tile_addr = [&](int s, int q) { return base + (uint32_t)(s * NT + q) * TC_TILE_BYTES; };
    auto failed = [&]() { return *(volatile int *)&fail_s != 0; };

    if (warp == TMA_PROD_WARP) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int it = 0;
            // operands of a tile: both maps, their row coordinates, k-blocks
            struct Ops {
                const CUtensorMap *ma, *mb;
                int rowa, rowb, nk, pair;
            };
            auto ops_of = [&](int ti) {
                const int4 tl = tiles[ti];
                const GemmTask t = tasks[tl.x];
                const bool trsm = (t.flags & 64) != 0;
                const int mb = mapidx[t.c];
                Ops o;
                o.ma = maps + mb + ((t.flags & 1) ? TMAP_U : TMAP_L);
                o.mb = maps + mb + (trsm ? ((t.flags & 128) ? TMAP_I2 : TMAP_I) : ((t.flags & 2) ? TMAP_U : TMAP_L));
                o.rowa = t.arow0 + tl.y * TC_BM;
                o.rowb = (trsm ? 0 : m.browoff[t.b]) + tl.z * TC_BN;
                o.nk = (m.width[t.c] + TC_BK - 1) / TC_BK;
                o.pair = tl.w & 1;
                return o;
            };
            Ops nxt{};
            if (blockIdx.x < ntiles) nxt = ops_of(blockIdx.x);
            for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x) {
                const Ops o = nxt;
                if (ti + (int)gridDim.x < ntiles) nxt = ops_of(ti + gridDim.x);   // in flight during this tile
                const CUtensorMap *ma = o.ma, *mbm = o.mb;
                const int rowa = o.rowa, rowb = o.rowb, nk = o.nk;
                const uint32_t bytes = (o.pair ? 3u : 2u) * BOX_BYTES;
                bool ok = true;
                for (int kb = 0; kb < nk; kb++, it++) {
                    const int s = it % S;
                    if (it >= S && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((it / S - 1) & 1))) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(smem_u32(&full[s]), bytes);
                    tma_load_3d(tile_addr(s, 0), ma, kb * TC_BK, rowa, 0, smem_u32(&full[s]));
                    if (o.pair) tma_load_3d(tile_addr(s, QA1), ma, kb * TC_BK, rowa + TC_BM, 0, smem_u32(&full[s]));
                    tma_load_3d(tile_addr(s, QB), mbm, kb * TC_BK, rowb, 0, smem_u32(&full[s]));
                }
                if (!ok) {
                    atomicExch(&fail_s, 1);
                    break;
                }
            }
            if (failed()) {
                // the loads still in flight land before the CTA leaves
                for (int j = 1; j <= S && it - j >= 0; j++) {
                    const int k = it - j;
                    mbar_wait(smem_u32(&full[k % S]), (uint32_t)((k / S) & 1));
                }
            }
        }
    } else if (warp == TMA_MMA_WARP) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int it = 0, tl = 0;
            TcTileView nv{};
            if (blockIdx.x < ntiles) nv = tc_tile_view(m, tiles[blockIdx.x], tasks, coefL, coefU, nullptr);
            for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x, tl++) {
                const TcTileView v = nv;
                if (ti + (int)gridDim.x < ntiles)   // the next tile's view loads while this one runs
                    nv = tc_tile_view(m, tiles[ti + gridDim.x], tasks, coefL, coefU, nullptr);
                const uint32_t idesc = tc_idesc(tc_mma_n(v.ncols));
                const int ab = tl & 1;
                const uint32_t acc = tmem + (uint32_t)(ab * 256), acc1 = acc + 128u;
                const bool pair = v.pair != 0;
                if (tl >= 2 && !mbar_wait(smem_u32(&acce[ab]), (uint32_t)((tl / 2 - 1) & 1))) {
                    atomicExch(&fail_s, 1);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                bool ok = true;
                for (int kb = 0; kb < v.nk; kb++, it++) {
                    const int s = it % S;
                    if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((it / S) & 1))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 8; kk++) {
                        const uint32_t first = (kb > 0 || kk > 0) ? 1u : 0u;
                        if (SPLIT) {
                            const uint64_t bh = tc_sdesc(tile_addr(s, QB) + kk * 32),
                                           bl = tc_sdesc(tile_addr(s, QB + 1) + kk * 32);
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                if (h == 1 && !pair) break;
                                const uint64_t ah = tc_sdesc(tile_addr(s, h * QA1) + kk * 32),
                                               al = tc_sdesc(tile_addr(s, h * QA1 + 1) + kk * 32);
                                const uint32_t ac = h ? acc1 : acc;
                                tc_mma(ac, al, bh, idesc, first);
                                tc_mma(ac, ah, bl, idesc, 1u);
                                tc_mma(ac, ah, bh, idesc, 1u);
                            }
                        } else {
                            const uint64_t bd = tc_sdesc(tile_addr(s, QB) + kk * 32);
                            tc_mma(acc, tc_sdesc(tile_addr(s, 0) + kk * 32), bd, idesc, first);
                            if (pair) tc_mma(acc1, tc_sdesc(tile_addr(s, QA1) + kk * 32), bd, idesc, first);
                        }
                    }
                    tc_commit(smem_u32(&empty[s]));
                }
                if (!ok) {
                    atomicExch(&fail_s, 1);
                    break;
                }
                tc_commit(smem_u32(&accf[ab]));
            }
            tc_commit(smem_u32(&drained));
            if (!mbar_wait(smem_u32(&drained), 0u)) atomicExch(&fail_s, 1);
        }
    } else {
        // ---------------- epilogue (warps 0-3) ----------------
        float *E = epi + warp * 32 * 33;
        int tl = 0;
        for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x, tl++) {
            const TcTileView v = tc_tile_view(m, tiles[ti], tasks, coefL, coefU, nullptr);
            const int ab = tl & 1;
            const int myrow = warp * 32 + lane;
            const bool trsm = (v.flags & 64) != 0;
            const int nh = v.pair ? 2 : 1;
            int tr[2] = {-1, -1};
            for (int h = 0; h < nh; h++) {
                const int row = h * TC_BM + myrow;     // row of the pair, from the first tile's first row
                if (row < v.M - v.i0 && !trsm)
                    tr[h] = panel_row_of(m, v.f, m.rowidx[m.rowbase[v.c] + v.arow + row]);
            }
            if (!mbar_wait(smem_u32(&accf[ab]), (uint32_t)((tl / 2) & 1))) {
                atomicExch(&fail_s, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            trow_s[0][myrow] = tr[0];
            trow_s[1][myrow] = tr[1];
            __syncwarp();
            float *C = ((v.flags & 4) ? coefU : coefL) + m.coefoff[v.f];
            const int ldf = m.ld[v.f], wf = m.width[v.f];
            const int tcol0 = m.bfrow[v.b] + v.j0 - m.fcol[v.f];
            const bool lower_only = (v.flags & 8) != 0;
            for (int h = 0; h < nh; h++)
            for (int cb = 0; cb < TC_BN; cb += 32) {
                const int mrows = min(TC_BM, v.M - v.i0 - h * TC_BM);   // valid rows of this half
                uint32_t r[32];
                tc_ld32(tmem + (uint32_t)(ab * 256 + h * 128) + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, r);
                __syncwarp();
#pragma unroll
                for (int q = 0; q < 32; q++) E[lane * 33 + q] = __uint_as_float(r[q]);
                __syncwarp();
                const int j = cb + lane;
                if (j < v.ncols && trsm) {
                    const int ldc = m.ld[v.c];
                    float *O = scr + v.out + (int64_t)(v.i0 + h * TC_BM) * ldc + v.j0;
                    for (int rr = 0; rr < 32; rr++) {
                        const int i = warp * 32 + rr;
                        if (i >= mrows) break;
                        O[(int64_t)i * ldc + j] = E[rr * 33 + lane];
                    }
                } else if (!trsm && cb < v.ncols) {
                    const int nvalid = min(32, v.ncols - cb);
                    const int tcs = tcol0 + cb, a0 = tcs & ~3, o = tcs - a0;
                    for (int k = lane; k < 32 * 9; k += 32) {
                        const int rr = k / 9, g = k - rr * 9;
                        const int t2 = trow_s[h][warp * 32 + rr];
                        if (t2 < 0) continue;
                        float a[4];
                        bool any = false;
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            const int jj = 4 * g + u - o, tc = a0 + 4 * g + u;
                            const bool ok = jj >= 0 && jj < nvalid && !(lower_only && t2 < wf && tc > t2);
                            a[u] = ok ? -E[rr * 33 + (ok ? jj : 0)] : 0.f;
                            any |= ok;
                        }
                        if (any) red_add_v4(&C[(int64_t)t2 * ldf + a0 + 4 * g], a[0], a[1], a[2], a[3]);
                    }
                }
                __syncwarp();
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&acce[ab]));
        }
    }
    if (tid == 0 && failed()) atomicAdd(&st->timeout, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == TMA_MMA_WARP) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMA_TMEM_COLS)
                     : "memory");
    }
}

// hi / lo split of panel rows for the TMA operands: rows [r0, r0 + 32) of
// cblk c's panel (L, or U^t when the job's panel flag is set), w columns, into
// hilo[0][...] = tf32(x) and hilo[ncoef][...] = x - tf32(x), same offsets as
// the coeftab.  Jobs: {cblk, first row, panel, -}.
__global__ void k_split_rows(Meta m, const int4 *__restrict__ jobs, const float *__restrict__ coefL,
                             const float *__restrict__ coefU, float *__restrict__ hilo, int64_t ncoef,
                             int64_t coefnbr) {
    const int4 jb = jobs[blockIdx.x];
    const int c = jb.x, r0 = jb.y;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int nr = min(32, h - r0);
    const int64_t off = m.coefoff[c] + (jb.z ? coefnbr : 0) + (int64_t)r0 * ld;
    const float *src = (jb.z ? coefU : coefL) + m.coefoff[c] + (int64_t)r0 * ld;
    float *hi = hilo + off, *lo = hilo + ncoef + off;
    const int wv = (w + 3) >> 2;   // float4 per row (the panel's rows are 16-byte aligned, ld % 4 == 0)
    for (int e = threadIdx.x; e < nr * wv; e += blockDim.x) {
        const int i = e / wv, q = e - i * wv;
        const float4 x = reinterpret_cast<const float4 *>(src + (int64_t)i * ld)[q];
        float4 h4, l4;
        h4.x = tf32_hi(x.x); h4.y = tf32_hi(x.y); h4.z = tf32_hi(x.z); h4.w = tf32_hi(x.w);
        l4.x = x.x - h4.x; l4.y = x.y - h4.y; l4.z = x.z - h4.z; l4.w = x.w - h4.w;
        reinterpret_cast<float4 *>(hi + (int64_t)i * ld)[q] = h4;
        reinterpret_cast<float4 *>(lo + (int64_t)i * ld)[q] = l4;
    }
}

}  // namespace pgpu
