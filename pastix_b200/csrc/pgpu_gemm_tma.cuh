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
// Roles (320 threads, one CTA per SM walking the level's tiles):
//   warps 0-3, 6-9: epilogue (TMEM -> registers -> a swizzled 32 x 32 shared
//              buffer per warp -> 16-byte vector reductions along the target
//              rows);
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
#include <cuda_fp16.h>
#include <type_traits>

#include "pgpu_common.cuh"
#include "pgpu_factor.cuh"
#include "pgpu_gemm_tc.cuh"

namespace pgpu {

// warps 0-3 and 6-9 write back the accumulators (two warps per TMEM lane
// quarter, each taking every other 32-column chunk), warp 4 loads, warp 5
// issues the MMAs
constexpr int TMA_THREADS = 320, TMA_EPI_WARPS = 8;
constexpr int TMA_PROD_WARP = 4, TMA_MMA_WARP = 5;
constexpr int TMA_EPI_BYTES = TMA_EPI_WARPS * 32 * 32 * 4;   // a swizzled 32 x 32 float buffer per warp
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
    return TmaCfg<SPLIT>::STAGES * TmaCfg<SPLIT>::TILES * TC_TILE_BYTES + TMA_EPI_BYTES + 1024;
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

// Everything the three roles need for one tile, built on the host when the
// plan is made: the kernel reads one 96-byte record per tile (loaded one or
// two tiles ahead) instead of walking tile -> task -> cblk tables through
// chains of dependent loads before it can issue a tile's loads or MMAs.
struct __align__(16) TcDesc {
    int mapa, mapb, rowa, rowb;   // tensor maps (indices into maps) and row coordinates of A and B
    int nk, ncols, pair, flags;   // k-blocks, valid columns, paired 128-row tiles, task flags (64: TRSM)
    int mrows, ldo, wf, tcol;     // rows from the tile's first; target (or output) row stride, target
                                  // cblk width (lower-triangle rule), first target column
    int pad[4];
    int64_t off;                  // target panel offset from coefL, or (TRSM) output offset in scr
    int64_t rmap;                 // row-map index of the tile's first row (update tiles)
    int64_t sa, sb;               // 3xFP16: scale index of the first A row, of the first B row
};
static_assert(sizeof(TcDesc) == 96, "TcDesc is six 16-byte vectors");

__device__ __forceinline__ TcDesc tc_desc_load(const TcDesc *p) {
    TcDesc d;
    const int4 *s = reinterpret_cast<const int4 *>(p);
    int4 *o = reinterpret_cast<int4 *>(&d);
#pragma unroll
    for (int k = 0; k < 6; k++) o[k] = __ldg(s + k);
    return d;
}

// F16 (with SPLIT): "3xFP16" operands -- every row r of a source matrix
// (panel rows, diagonal-block inverse rows) is scaled by a power of two
// 2^e_r that brings its largest magnitude into [2^14, 2^15), then split into
// hi = fp16(x 2^e_r) and lo = fp16(x 2^e_r - hi) (both round to nearest):
// 11 + 11 significant bits, the precision of the 3xTF32 split, in half the
// bytes, on the FP16 MMA rate (twice the TF32 rate).  The k-block is 64
// halves (128 bytes, the same SWIZZLE_128B tile as 32 floats) and each MMA
// covers K = 16.  The epilogue multiplies the accumulator by the rows'
// inverse scales 2^-e_a 2^-e_b (hscale, one float per source row; hsbase
// gives each operand map's first row there), exact powers of two.
template <bool SPLIT, bool F16 = false>
__global__ void __launch_bounds__(TMA_THREADS, 1)
    k_gemm_scatter_tc_tma(const TcDesc *__restrict__ desc, int ntiles, float *__restrict__ coefL, Status *st,
                          float *__restrict__ scr, const CUtensorMap *__restrict__ maps,
                          const int *__restrict__ tmap, const float *__restrict__ hscale = nullptr) {
    static_assert(!F16 || SPLIT, "the FP16 operands are always split");
    constexpr int S = TmaCfg<SPLIT>::STAGES, NT = TmaCfg<SPLIT>::TILES, PL = TmaCfg<SPLIT>::PL;
    constexpr int BK = F16 ? 64 : TC_BK;                              // elements per k-block (128 B per row)
    constexpr uint32_t BOX_BYTES = (uint32_t)PL * TC_TILE_BYTES;   // one operand box (hi [+ lo])
    constexpr int QA1 = PL, QB = 2 * PL;                            // tile slots of A1 and B in a stage
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t full[S], empty[S], accf[2], acce[2], drained;
    __shared__ uint32_t tmem_base_s;
    __shared__ int fail_s;

    const uint32_t raw = smem_u32(tc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char *sbase = tc_smem_raw + (base - raw);
    float *epi = reinterpret_cast<float *>(sbase + S * NT * TC_TILE_BYTES);   // [8][32][32]

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
            mbar_init(smem_u32(&acce[b]), TMA_EPI_WARPS);
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
            TcDesc nx{};
            if (blockIdx.x < ntiles) nx = tc_desc_load(desc + blockIdx.x);
            for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x) {
                const TcDesc o = nx;
                if (ti + (int)gridDim.x < ntiles) nx = tc_desc_load(desc + ti + gridDim.x);   // for the next tile
                const CUtensorMap *ma = maps + o.mapa, *mbm = maps + o.mapb;
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
                    tma_load_3d(tile_addr(s, 0), ma, kb * BK, rowa, 0, smem_u32(&full[s]));
                    if (o.pair) tma_load_3d(tile_addr(s, QA1), ma, kb * BK, rowa + TC_BM, 0, smem_u32(&full[s]));
                    tma_load_3d(tile_addr(s, QB), mbm, kb * BK, rowb, 0, smem_u32(&full[s]));
                }
                if (!ok) {
                    atomicExch(&fail_s, 1);
                    break;
                }
            }
            if (failed()) {
                // the loads still in flight land before the CTA leaves; if one
                // of these waits gives up as well, the CTA may leave with bulk
                // copies still writing its shared memory: recorded apart, and the
                // host treats the whole factorization as failed
                for (int j = 1; j <= S && it - j >= 0; j++) {
                    const int k = it - j;
                    if (!mbar_wait(smem_u32(&full[k % S]), (uint32_t)((k / S) & 1))) atomicAdd(&st->drain_timeout, 1);
                }
            }
        }
    } else if (warp == TMA_MMA_WARP) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int it = 0, tl = 0;
            TcDesc nx{};
            if (blockIdx.x < ntiles) nx = tc_desc_load(desc + blockIdx.x);
            for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x, tl++) {
                const TcDesc v = nx;
                if (ti + (int)gridDim.x < ntiles) nx = tc_desc_load(desc + ti + gridDim.x);   // for the next tile
                const uint32_t idesc = F16 ? tc_idesc_f16(tc_mma_n(v.ncols)) : tc_idesc(tc_mma_n(v.ncols));
                const int vnk = v.nk;
                const int ab = tl & 1;
                const uint32_t acc = tmem + (uint32_t)(ab * 256), acc1 = acc + 128u;
                const bool pair = v.pair != 0;
                if (tl >= 2 && !mbar_wait(smem_u32(&acce[ab]), (uint32_t)((tl / 2 - 1) & 1))) {
                    atomicExch(&fail_s, 1);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                bool ok = true;
                for (int kb = 0; kb < vnk; kb++, it++) {
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
                                if (F16) {
                                    tc_mma_f16(ac, al, bh, idesc, first);
                                    tc_mma_f16(ac, ah, bl, idesc, 1u);
                                    tc_mma_f16(ac, ah, bh, idesc, 1u);
                                } else {
                                    tc_mma(ac, al, bh, idesc, first);
                                    tc_mma(ac, ah, bl, idesc, 1u);
                                    tc_mma(ac, ah, bh, idesc, 1u);
                                }
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
        // ---------------- epilogue (warps 0-3 and 6-9) ----------------
        // The next tile's view, target rows and row scales are loaded while
        // the current tile is written back (prep of tile t + 1 before the
        // wait on tile t's accumulator): the epilogue's per-tile load chains
        // stay off the path of the reductions.
        const int ew = warp < 4 ? warp : warp - 2;   // epilogue warp 0..7
        const int qw = warp & 3;                       // TMEM lane quarter (rows 32 qw .. 32 qw + 31)
        const int grp = warp < 4 ? 0 : 1;              // column chunks 32 grp, 32 grp + 64
        float *E = epi + ew * 32 * 32;
        const int myrow = qw * 32 + lane;
        // two stages: the descriptor of tile t + 2 is loaded while tile t is
        // written back, and the row targets / scales of tile t + 1 (which need
        // its descriptor) are requested then too
        struct EpiTile {
            TcDesc d;
            int tr[2];
            float rs[2], cs[2];
        };
        auto prep = [&](const TcDesc &d, EpiTile &e) {
            e.d = d;
            const bool trsm = (d.flags & 64) != 0;
            for (int h = 0; h < 2; h++) {
                const int row = h * TC_BM + myrow;   // row of the pair, from the first tile's first row
                const bool ok = (h == 0 || d.pair) && row < d.mrows;
                e.tr[h] = (ok && !trsm) ? tmap[d.rmap + row] : -1;
                e.rs[h] = (F16 && ok) ? hscale[d.sa + row] : 1.f;
                // this warp's two 32-column chunks: column 32 grp + 64 h + lane
                const int col = 32 * grp + 64 * h + lane;
                e.cs[h] = (F16 && col < d.ncols) ? hscale[d.sb + col] : 0.f;
            }
        };
        EpiTile cur{}, nxt{};
        TcDesc dn{};
        if (blockIdx.x < ntiles) prep(tc_desc_load(desc + blockIdx.x), cur);
        if (blockIdx.x + (int)gridDim.x < ntiles) dn = tc_desc_load(desc + blockIdx.x + gridDim.x);
        int tl = 0;
        for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x, tl++) {
            if (ti + (int)gridDim.x < ntiles) {
                prep(dn, nxt);
                if (ti + 2 * (int)gridDim.x < ntiles) dn = tc_desc_load(desc + ti + 2 * gridDim.x);
            }
            const TcDesc &v = cur.d;
            const int ab = tl & 1;
            const bool trsm = (v.flags & 64) != 0;
            const int nh = v.pair ? 2 : 1;
            if (!mbar_wait(smem_u32(&accf[ab]), (uint32_t)((tl / 2) & 1))) {
                atomicExch(&fail_s, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int trw[2] = {cur.tr[0], cur.tr[1]};   // each lane's row target, shuffled to the writers
            const float rs[2] = {cur.rs[0], cur.rs[1]};
            const float csr[2] = {cur.cs[0], cur.cs[1]};
            float *C = coefL + v.off;
            const int ldf = v.ldo, wf = v.wf;
            const int tcol0 = v.tcol;
            const bool lower_only = (v.flags & 8) != 0;
            // the update subtracts: the sign rides on the row scale
            const float sgn = trsm ? 1.f : -1.f;
            for (int h = 0; h < nh; h++)
            for (int cb = 32 * grp; cb < TC_BN; cb += 64) {
                const int mrows = min(TC_BM, v.mrows - h * TC_BM);   // valid rows of this half
                uint32_t r[32];
                tc_ld32(tmem + (uint32_t)(ab * 256 + h * 128) + ((uint32_t)(qw * 32) << 16) + (uint32_t)cb, r);
                __syncwarp();
                // this lane's row (TMEM lane) as eight 16-byte groups, group g at
                // slot g ^ (row & 7): conflict-free both for the row-wise stores
                // here and for the loads along a row / down a column below
                float x[32];
                if (F16) {
                    // column cb + lane's inverse scale (loaded with the tile), broadcast column by column
                    const float cs = (cb - 32 * grp) ? csr[1] : csr[0], rsh = (h ? rs[1] : rs[0]) * sgn;
#pragma unroll
                    for (int q = 0; q < 32; q++) x[q] = __uint_as_float(r[q]) * rsh * __shfl_sync(0xffffffffu, cs, q);
                } else {
#pragma unroll
                    for (int q = 0; q < 32; q++) x[q] = __uint_as_float(r[q]) * sgn;
                }
#pragma unroll
                for (int g = 0; g < 8; g++)
                    *reinterpret_cast<float4 *>(E + lane * 32 + ((g ^ (lane & 7)) << 2)) =
                        make_float4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]);
                __syncwarp();
                const int j = cb + lane;
                if (j < v.ncols && trsm) {
                    const int ldc = v.ldo;
                    float *O = scr + v.off + (int64_t)h * TC_BM * ldc;
                    for (int rr = 0; rr < 32; rr++) {
                        const int i = qw * 32 + rr;
                        if (i >= mrows) break;
                        O[(int64_t)i * ldc + j] = E[rr * 32 + ((((lane >> 2) ^ (rr & 7)) << 2) | (lane & 3))];
                    }
                } else if (!trsm && cb < v.ncols) {
                    const int nvalid = min(32, v.ncols - cb);
                    const int tcs = tcol0 + cb, a0 = tcs & ~3;
                    const int trh = h ? trw[1] : trw[0];
                    // target group g (columns a0 + 4 g ..) takes source columns 4 g - O ..
                    // 4 g + 3 - O: the tail of group g - 1 and the head of group g, the
                    // offset O = tcs mod 4 a compile-time constant per branch
                    auto reduce = [&](auto oc) {
                        constexpr int O = decltype(oc)::value;
                        for (int k = lane; k < 32 * 9; k += 32) {
                            const int rr = k / 9, g = k - rr * 9;
                            const int t2 = __shfl_sync(0xffffffffu, trh, rr);
                            if (t2 < 0 || (O == 0 && g == 8)) continue;
                            const float *Er = E + rr * 32;
                            const int sw = rr & 7;
                            float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
                            if (O > 0 && g >= 1) lo = *reinterpret_cast<const float4 *>(Er + (((g - 1) ^ sw) << 2));
                            if (g <= 7) hi = *reinterpret_cast<const float4 *>(Er + ((g ^ sw) << 2));
                            float a[4];
                            if (O == 0) { a[0] = hi.x; a[1] = hi.y; a[2] = hi.z; a[3] = hi.w; }
                            if (O == 1) { a[0] = lo.w; a[1] = hi.x; a[2] = hi.y; a[3] = hi.z; }
                            if (O == 2) { a[0] = lo.z; a[1] = lo.w; a[2] = hi.x; a[3] = hi.y; }
                            if (O == 3) { a[0] = lo.y; a[1] = lo.z; a[2] = lo.w; a[3] = hi.x; }
                            const int j0 = 4 * g - O;   // source column of a[0]
                            if (j0 < 0 || j0 + 3 >= nvalid || lower_only) {
                                bool any = false;
#pragma unroll
                                for (int u = 0; u < 4; u++) {
                                    const int jj = j0 + u, tc = a0 + 4 * g + u;
                                    const bool ok = jj >= 0 && jj < nvalid && !(lower_only && t2 < wf && tc > t2);
                                    a[u] = ok ? a[u] : 0.f;
                                    any |= ok;
                                }
                                if (!any) continue;
                            }
                            red_add_v4(&C[(int64_t)t2 * ldf + a0 + 4 * g], a[0], a[1], a[2], a[3]);
                        }
                    };
                    switch (tcs - a0) {
                        case 0: reduce(std::integral_constant<int, 0>{}); break;
                        case 1: reduce(std::integral_constant<int, 1>{}); break;
                        case 2: reduce(std::integral_constant<int, 2>{}); break;
                        default: reduce(std::integral_constant<int, 3>{}); break;
                    }
                }
                __syncwarp();
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&acce[ab]));
            cur = nxt;
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

// ---------------------------------------------------------------------------
// 3xFP16 operands: per-row power-of-two scaling and hi / lo split.
//
// Row scale: the largest magnitude m of the row has binary exponent E
// (2^E <= m < 2^(E+1)); e = 14 - E puts it in [2^14, 2^15), below the FP16
// maximum 65504 and far above its normal minimum 2^-14.  e is clamped to
// [-126, 126] so that 2^e and 2^-e are normal floats (an all-zero row keeps
// e = 0).  The row's stored scale is 2^-e, which the GEMM epilogue applies.
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

// One warp splits one row of w floats (src 16-byte aligned when w >= 4):
// optional FP32 copy to dst, hi / lo halves at hi and hi + hplane, the
// inverse scale at *sc.
__device__ __forceinline__ void split_row_h16(const float *__restrict__ src, int w, float *__restrict__ dst,
                                              __half *__restrict__ hi, int64_t hplane, float *__restrict__ sc,
                                              int lane) {
    const int wv = w >> 2;
    constexpr int RV = 4;   // rows of up to 32 RV float4 stay in registers: read once, all loads in flight
    if (wv <= 32 * RV) {
        float4 x[RV];
        float mx = 0.f;
#pragma unroll
        for (int u = 0; u < RV; u++) {
            const int q = lane + 32 * u;
            x[u] = q < wv ? __ldg(reinterpret_cast<const float4 *>(src) + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        const int jt = 4 * wv + lane;   // the tail (w % 4 columns), one per lane
        const float xt = jt < w ? src[jt] : 0.f;
#pragma unroll
        for (int u = 0; u < RV; u++)
            mx = fmaxf(mx, fmaxf(fmaxf(fabsf(x[u].x), fabsf(x[u].y)), fmaxf(fabsf(x[u].z), fabsf(x[u].w))));
        mx = fmaxf(mx, fabsf(xt));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        int e = 0;
        if (mx > 0.f) {
            const int E = ((__float_as_int(mx) >> 23) & 0xff) - 127;
            e = max(-126, min(126, 14 - E));
        }
        const float s = pow2f(e);
        if (lane == 0) *sc = pow2f(-e);
        __half *lo = hi + hplane;
#pragma unroll
        for (int u = 0; u < RV; u++) {
            const int q = lane + 32 * u;
            if (q < wv) {
                if (dst) reinterpret_cast<float4 *>(dst)[q] = x[u];
                const float y[4] = {x[u].x * s, x[u].y * s, x[u].z * s, x[u].w * s};
                __half h[4], l[4];
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    h[v] = __float2half_rn(y[v]);
                    l[v] = __float2half_rn(y[v] - __half2float(h[v]));
                }
                reinterpret_cast<__half2 *>(hi)[2 * q] = __halves2half2(h[0], h[1]);
                reinterpret_cast<__half2 *>(hi)[2 * q + 1] = __halves2half2(h[2], h[3]);
                reinterpret_cast<__half2 *>(lo)[2 * q] = __halves2half2(l[0], l[1]);
                reinterpret_cast<__half2 *>(lo)[2 * q + 1] = __halves2half2(l[2], l[3]);
            }
        }
        if (jt < w) {
            if (dst) dst[jt] = xt;
            const float y = xt * s;
            const __half h = __float2half_rn(y);
            hi[jt] = h;
            lo[jt] = __float2half_rn(y - __half2float(h));
        }
        return;
    }
    float mx = 0.f;
    for (int q = lane; q < wv; q += 32) {
        const float4 x = reinterpret_cast<const float4 *>(src)[q];
        mx = fmaxf(mx, fmaxf(fmaxf(fabsf(x.x), fabsf(x.y)), fmaxf(fabsf(x.z), fabsf(x.w))));
    }
    for (int j = 4 * wv + lane; j < w; j += 32) mx = fmaxf(mx, fabsf(src[j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int e = 0;
    if (mx > 0.f) {
        const int E = ((__float_as_int(mx) >> 23) & 0xff) - 127;
        e = max(-126, min(126, 14 - E));
    }
    const float s = pow2f(e);
    if (lane == 0) *sc = pow2f(-e);
    __half *lo = hi + hplane;
    for (int q = lane; q < wv; q += 32) {
        const float4 x = reinterpret_cast<const float4 *>(src)[q];
        if (dst) reinterpret_cast<float4 *>(dst)[q] = x;
        const float y[4] = {x.x * s, x.y * s, x.z * s, x.w * s};
        __half h[4], l[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            h[u] = __float2half_rn(y[u]);
            l[u] = __float2half_rn(y[u] - __half2float(h[u]));
        }
        reinterpret_cast<__half2 *>(hi)[2 * q] = __halves2half2(h[0], h[1]);
        reinterpret_cast<__half2 *>(hi)[2 * q + 1] = __halves2half2(h[2], h[3]);
        reinterpret_cast<__half2 *>(lo)[2 * q] = __halves2half2(l[0], l[1]);
        reinterpret_cast<__half2 *>(lo)[2 * q + 1] = __halves2half2(l[2], l[3]);
    }
    for (int j = 4 * wv + lane; j < w; j += 32) {
        const float x = src[j];
        if (dst) dst[j] = x;
        const float y = x * s;
        const __half h = __float2half_rn(y);
        hi[j] = h;
        lo[j] = __float2half_rn(y - __half2float(h));
    }
}

// Target rows of the tensor-core update tasks, once per plan: for task
// tlist[blockIdx.x] and each row i of its M rows, the panel row of the facing
// cblk that source row arow0 + i lands in (kernels/core_zgemmsp.c:170-250
// walks the facing blocks for this).  tmap[taux[3 task] + i].
__global__ void k_task_rowmap(Meta m, const GemmTask *__restrict__ tasks, const int *__restrict__ tlist,
                              const int64_t *__restrict__ taux, int *__restrict__ tmap) {
    const int id = tlist[blockIdx.x];
    const GemmTask t = tasks[id];
    const int64_t base = taux[3 * (int64_t)id];
    const int *rows = m.rowidx + m.rowbase[t.c] + t.arow0;
    for (int i = threadIdx.x; i < t.M; i += blockDim.x) tmap[base + i] = panel_row_of(m, t.f, rows[i]);
}

// Layout of the FP16 planes: per operand map (mapidx[c] + kind) the first
// element in the planes (hoff, rows of ld16 = round_up(w_c, 8) halves) and the
// first row in hscale (hsbase).
__host__ __device__ inline int ld16_of(int w) { return (w + 7) & ~7; }

// Split jobs {cblk, first row, kind (TMAP_*), -}: rows [r0, r0 + 32) of the
// source matrix of that kind (L / U panel rows, or the rows of the first /
// second diagonal-block inverse), one warp per row.
__global__ void __launch_bounds__(256) k_split_rows_h16(Meta m, const int4 *__restrict__ jobs,
                                                        const float *__restrict__ coefL,
                                                        const float *__restrict__ coefU,
                                                        const float *__restrict__ inv, __half *__restrict__ h16,
                                                        int64_t hplane, float *__restrict__ hscale,
                                                        const int64_t *__restrict__ hoff,
                                                        const int64_t *__restrict__ hsbase,
                                                        const int *__restrict__ mapidx) {
    const int4 jb = jobs[blockIdx.x];
    const int c = jb.x, r0 = jb.y, kind = jb.z;
    const int w = m.width[c], ld = m.ld[c], l16 = ld16_of(w);
    const int rows = kind < TMAP_I ? m.height[c] : w;
    const float *src = kind == TMAP_L ? coefL + m.coefoff[c]
                       : kind == TMAP_U ? coefU + m.coefoff[c]
                                        : inv + m.invoff[c] + (kind == TMAP_I2 ? inv_span(w, ld) : 0);
    const int mi = mapidx[c] + kind;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r1 = min(r0 + 32, rows);
    for (int i = r0 + warp; i < r1; i += blockDim.x >> 5)
        split_row_h16(src + (int64_t)i * ld, w, nullptr, h16 + hoff[mi] + (int64_t)i * l16, hplane,
                      hscale + hsbase[mi] + i, lane);
}

// TRSM copy-back with the FP16 split: rows [r0, r0 + 32) of the level's
// TRSM output (chunks {cblk, r0, side, -} as k_trsm_copyback) into the panel
// and, when the cblk is a tensor-core source, into its FP16 planes.
__global__ void __launch_bounds__(256) k_trsm_copyback_h16(Meta m, const int4 *__restrict__ chunks,
                                                           const int64_t *__restrict__ scroff,
                                                           const float *__restrict__ scr, float *__restrict__ coefL,
                                                           float *__restrict__ coefU, __half *__restrict__ h16,
                                                           int64_t hplane, float *__restrict__ hscale,
                                                           const int64_t *__restrict__ hoff,
                                                           const int64_t *__restrict__ hsbase,
                                                           const int *__restrict__ mapidx) {
    const int4 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c], l16 = ld16_of(w);
    const int nr = min(32, h - r0);
    const float *src = scr + scroff[c] + (ch.z ? inv_span(h - w, ld) : 0) + (int64_t)(r0 - w) * ld;
    float *dst = (ch.z ? coefU : coefL) + m.coefoff[c] + (int64_t)r0 * ld;
    const int mb = mapidx[c];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (mb < 0) {   // not a tensor-core source: the FP32 rows only
        for (int e = threadIdx.x; e < nr * w; e += blockDim.x) {
            const int i = e / w, j = e - i * w;
            dst[(int64_t)i * ld + j] = src[(int64_t)i * ld + j];
        }
        return;
    }
    const int mi = mb + (ch.z ? TMAP_U : TMAP_L);
    for (int i = warp; i < nr; i += blockDim.x >> 5)
        split_row_h16(src + (int64_t)i * ld, w, dst + (int64_t)i * ld, h16 + hoff[mi] + (int64_t)(r0 + i) * l16,
                      hplane, hscale + hsbase[mi] + r0 + i, lane);
}

}  // namespace pgpu
