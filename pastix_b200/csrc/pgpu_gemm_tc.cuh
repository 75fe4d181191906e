// Update GEMM with indexed scatter-add on the 5th-generation tensor cores
// (tcgen05, sm_100a) for the single-precision factorization: C = A B^T with
// A = panel rows [arow0 + i0, +128) of cblk c, B = rows [browoff_b + j0, +128)
// of block b, K = w_c, FP32 accumulation in TMEM; C is subtracted from the
// facing cblk f at (panel row of the source row in f, frownum_b + j -
// fcolnum_f), as kernels/core_zgemmsp.c:104 core_zgemmsp_1d1d + core_zgeadd do.
//
// Two operand modes:
//   SPLIT = false: the FP32 operands are read as TF32 (one MMA per k-step);
//   SPLIT = true : "3xTF32" -- every operand is split into x = hi + lo with
//                  hi = tf32(x) (round to nearest) and lo = x - hi, and
//                  A B^T ~ lo_a hi_b + hi_a lo_b + hi_a hi_b (three MMAs per
//                  k-step, small terms first), which keeps about FP32 accuracy.
//
// Per CTA (128 threads, one 128 x 128 output tile):
//   * A and B k-blocks (128 rows x 32 floats = 128 B per row) are staged in
//     shared memory in the canonical K-major SWIZZLE_128B layout (8-row groups
//     of 1024 B, 16-byte chunk c of row r stored at chunk c ^ (r & 7)):
//     with cp.async TC_STAGES deep (TF32), or through registers where the
//     split happens, double-buffered with the next k-block's global loads in
//     flight while the current MMAs run (3xTF32);
//   * one thread issues the tcgen05.mma (K = 8 each) of a k-block and commits
//     them to the stage's mbarrier, which frees the stage;
//   * the accumulator (128 lanes x 128 fp32 columns of TMEM) is read back with
//     tcgen05.ld by the 4 warps (warp w owns lanes 32w..32w+31), transposed
//     through shared memory so a warp's atomics hit 32 consecutive columns.
// Every mbarrier wait is bounded; on time-out the CTA records the failure in
// Status::timeout, frees its TMEM and leaves the tile untouched.
#pragma once

#include "pgpu_common.cuh"
#include "pgpu_factor.cuh"

namespace pgpu {

constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 32, TC_THREADS = 128;
constexpr int TC_TILE_BYTES = TC_BM * TC_BK * 4;                     // 16 KB per operand tile
template <bool SPLIT> struct TcCfg;
template <> struct TcCfg<false> {
    static constexpr int STAGES = 3, TILES = 2;                        // A, B
};
template <> struct TcCfg<true> {
    static constexpr int STAGES = 2, TILES = 4;                        // A hi, A lo, B hi, B lo
};
template <bool SPLIT>
constexpr int tc_smem_bytes() {
    return TcCfg<SPLIT>::STAGES * TcCfg<SPLIT>::TILES * TC_TILE_BYTES + 1024;   // + alignment slack
}
constexpr int TC_TMEM_COLS = 128;


// Shared-memory matrix descriptor: K-major, SWIZZLE_128B, 8-row groups
// 1024 B apart (stride byte offset), version 1 (sm_100).
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(1u) << 16;                 // leading byte offset (unused, swizzled K-major)
    d |= static_cast<uint64_t>(1024u >> 4) << 32;         // stride byte offset
    d |= static_cast<uint64_t>(1u) << 46;                 // descriptor version
    d |= static_cast<uint64_t>(2u) << 61;                 // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D fp32, A/B tf32, both K-major, M = 128, N = n
// (a multiple of 16 up to 128: a tile with fewer valid columns issues
// narrower MMAs instead of multiplying zero rows).
__device__ __forceinline__ uint32_t tc_idesc(int n = TC_BN) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}
__device__ __forceinline__ int tc_mma_n(int ncols) { return min(TC_BN, (ncols + 15) & ~15); }
// The same for kind::f16 with FP16 A and B (format 0) and FP32 D.
__device__ __forceinline__ uint32_t tc_idesc_f16(int n = TC_BN) {
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}



__device__ __forceinline__ void tc_fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}

// kind::f16 (FP16 operands, K = 16 per instruction: 32 bytes of a 128-byte
// swizzled row, the same descriptor step as the TF32 form's K = 8).
__device__ __forceinline__ void tc_mma_f16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                           uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
          "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
          "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// The "hi" part of the 3xTF32 split (TF32 rounding, pgpu_common.cuh).
__device__ __forceinline__ float tf32_hi(float x) { return tf32_round(x); }

__device__ __forceinline__ void sts128(uint32_t saddr, float4 v) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(saddr), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}

template <bool SPLIT>
__global__ void __launch_bounds__(TC_THREADS) k_gemm_scatter_tc(Meta m, const int4 *__restrict__ tiles,
                                                                const GemmTask *__restrict__ tasks,
                                                                float *__restrict__ coefL,
                                                                float *__restrict__ coefU, Status *st,
                                                                const float *__restrict__ inv,
                                                                float *__restrict__ scr, int64_t *prof) {
    constexpr int S = TcCfg<SPLIT>::STAGES, NT = TcCfg<SPLIT>::TILES;
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t mbar[S];
    __shared__ uint32_t tmem_base_s;
    __shared__ int trow_s[TC_BM];
    __shared__ int fail_s;

    // 1024-byte aligned operand area (SWIZZLE_128B atoms)
    const uint32_t raw = smem_u32(tc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char *sbase = tc_smem_raw + (base - raw);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t t_start = prof ? global_ns() : 0;
    const int4 tl = tiles[blockIdx.x];
    const GemmTask t = tasks[tl.x];
    const int c = t.c, b = t.b, f = t.f;
    const int K = m.width[c], ld = m.ld[c];
    const bool trsm = (t.flags & 64) != 0;
    const int N = trsm ? K : m.blrow[b] - m.bfrow[b] + 1;
    const int i0 = tl.y * TC_BM, j0 = tl.z * TC_BN;
    const float *A = ((t.flags & 1) ? coefU : coefL) + m.coefoff[c] + (int64_t)(t.arow0 + i0) * ld;
    const float *B = trsm ? inv + m.invoff[c] + ((t.flags & 128) ? inv_span(K, ld) : 0) + (int64_t)j0 * ld
                          : ((t.flags & 2) ? coefU : coefL) + m.coefoff[c] + (int64_t)(m.browoff[b] + j0) * ld;
    const int mrows = min(TC_BM, t.M - i0), ncols = min(TC_BN, N - j0);
    const int nk = (K + TC_BK - 1) / TC_BK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S; s++) mbar_init(smem_u32(&mbar[s]), 1);
        fail_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        int tr = -1;
        if (tid < mrows && !trsm) tr = panel_row_of(m, f, m.rowidx[m.rowbase[c] + t.arow0 + i0 + tid]);
        trow_s[tid] = tr;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;

    // operand tile q (0 A / 1 B for TF32; 0 A hi, 1 A lo, 2 B hi, 3 B lo split) of stage s
    auto tile_addr = [&](int s, int q) { return base + (uint32_t)(s * NT + q) * TC_TILE_BYTES; };
    const int nmma = tc_mma_n(ncols);
    const uint32_t idesc = tc_idesc(nmma);
    auto issue = [&](int s, int kb) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int kk = 0; kk < TC_BK / 8; kk++) {
            const uint32_t first = (kb > 0 || kk > 0) ? 1u : 0u;
            if (SPLIT) {
                const uint64_t ah = tc_sdesc(tile_addr(s, 0) + kk * 32), al = tc_sdesc(tile_addr(s, 1) + kk * 32);
                const uint64_t bh = tc_sdesc(tile_addr(s, 2) + kk * 32), bl = tc_sdesc(tile_addr(s, 3) + kk * 32);
                tc_mma(tmem, al, bh, idesc, first);
                tc_mma(tmem, ah, bl, idesc, 1u);
                tc_mma(tmem, ah, bh, idesc, 1u);
            } else {
                tc_mma(tmem, tc_sdesc(tile_addr(s, 0) + kk * 32), tc_sdesc(tile_addr(s, 1) + kk * 32), idesc, first);
            }
        }
        tc_commit(smem_u32(&mbar[s]));
    };

    bool ok = true;
    if constexpr (!SPLIT) {
        auto load_stage = [&](int s, int kb) {
            const int k0 = kb * TC_BK;
            // 128 rows x 8 chunks of 16 B for each operand; 8 chunks per thread each
#pragma unroll
            for (int q = 0; q < (TC_BM * 8) / TC_THREADS; q++) {
                const int e = tid + q * TC_THREADS;
                const int r = e >> 3, ch = e & 7;
                const int kc = k0 + ch * 4;
                const uint32_t soff = (uint32_t)(r * 128 + ((ch ^ (r & 7)) << 4));
                const bool va = (r < mrows) && (kc < K);
                cp_async16(tile_addr(s, 0) + soff, va ? (const void *)(A + (int64_t)r * ld + kc) : (const void *)A,
                           va);
                const bool vb = (r < ncols) && (kc < K);
                if (r < nmma)
                    cp_async16(tile_addr(s, 1) + soff, vb ? (const void *)(B + (int64_t)r * ld + kc) : (const void *)B,
                               vb);
            }
        };
#pragma unroll
        for (int s = 0; s < S - 1; s++) {
            if (s < nk) load_stage(s, s);
            cp_async_commit();
        }
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % S;
            const int pk = kb + S - 1;
            if (pk < nk) {
                const int ps = pk % S;
                if (kb >= 1) {
                    // stage ps was last read by the MMAs of k-block kb-1
                    if (!mbar_wait(smem_u32(&mbar[ps]), (uint32_t)(((kb - 1) / S) & 1))) ok = false;
                }
                if (ok) load_stage(ps, pk);
            }
            cp_async_commit();
            cp_async_wait<S - 1>();
            tc_fence_async_smem();
            if (!__syncthreads_and(ok ? 1 : 0)) {
                ok = false;
                break;
            }
            if (tid == 0) issue(s, kb);
        }
    } else {
        // 3xTF32: global -> registers -> (hi, lo) -> swizzled shared memory
        constexpr int CH = (TC_BM * 8) / TC_THREADS;     // 8 chunks of 16 B per operand per thread
        float4 ra[CH], rb[CH];
        auto gload = [&](int kb) {
            const int k0 = kb * TC_BK;
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const int e = tid + q * TC_THREADS;
                const int r = e >> 3, ch = e & 7;
                const int kc = k0 + ch * 4;
                ra[q] = ((r < mrows) && (kc < K)) ? __ldg(reinterpret_cast<const float4 *>(A + (int64_t)r * ld + kc))
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
                rb[q] = ((r < ncols) && (kc < K)) ? __ldg(reinterpret_cast<const float4 *>(B + (int64_t)r * ld + kc))
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        };
        // (B rows >= nmma are stored too: the tile kernel keeps one code path)
        auto split_store = [&](int s) {
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const int e = tid + q * TC_THREADS;
                const int r = e >> 3, ch = e & 7;
                const uint32_t soff = (uint32_t)(r * 128 + ((ch ^ (r & 7)) << 4));
                float4 h, l;
                h.x = tf32_hi(ra[q].x); h.y = tf32_hi(ra[q].y); h.z = tf32_hi(ra[q].z); h.w = tf32_hi(ra[q].w);
                l.x = ra[q].x - h.x; l.y = ra[q].y - h.y; l.z = ra[q].z - h.z; l.w = ra[q].w - h.w;
                sts128(tile_addr(s, 0) + soff, h);
                sts128(tile_addr(s, 1) + soff, l);
                h.x = tf32_hi(rb[q].x); h.y = tf32_hi(rb[q].y); h.z = tf32_hi(rb[q].z); h.w = tf32_hi(rb[q].w);
                l.x = rb[q].x - h.x; l.y = rb[q].y - h.y; l.z = rb[q].z - h.z; l.w = rb[q].w - h.w;
                sts128(tile_addr(s, 2) + soff, h);
                sts128(tile_addr(s, 3) + soff, l);
            }
        };
        if (nk > 0) {
            gload(0);
            split_store(0);
        }
        tc_fence_async_smem();
        __syncthreads();
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb & 1;
            if (tid == 0) issue(s, kb);
            if (kb + 1 < nk) {
                gload(kb + 1);                       // in flight while the MMAs of kb run
                if (kb >= 1) {
                    // stage s^1 was last read by the MMAs of k-block kb-1
                    if (!mbar_wait(smem_u32(&mbar[s ^ 1]), (uint32_t)(((kb - 1) >> 1) & 1))) ok = false;
                }
                if (ok) split_store(s ^ 1);
                tc_fence_async_smem();
            }
            if (!__syncthreads_and(ok ? 1 : 0)) {
                ok = false;
                break;
            }
        }
    }
    // all MMAs done when the last commit's barrier flips
    if (ok && nk > 0) {
        if (!mbar_wait(smem_u32(&mbar[(nk - 1) % S]), (uint32_t)(((nk - 1) / S) & 1))) ok = false;
    }
    if constexpr (!SPLIT) cp_async_wait<0>();
    if (!ok) atomicExch(&fail_s, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!fail_s) {
        // epilogue: TMEM -> registers -> transpose in shared memory -> atomics
        float *E = reinterpret_cast<float *>(sbase) + warp * 32 * 33;
        float *O = trsm ? scr + t.out + (int64_t)i0 * ld + j0 : nullptr;
        float *C = ((t.flags & 4) ? coefU : coefL) + m.coefoff[f];
        const int ldf = m.ld[f], wf = m.width[f];
        const int tcol0 = m.bfrow[b] + j0 - m.fcol[f];
        const bool lower_only = (t.flags & 8) != 0;
        for (int cb = 0; cb < TC_BN; cb += 32) {
            uint32_t v[32];
            tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 32; q++) E[lane * 33 + q] = __uint_as_float(v[q]);
            __syncwarp();
            const int j = cb + lane;
            if (j < ncols && trsm) {
                for (int rr = 0; rr < 32; rr++) {
                    const int i = warp * 32 + rr;
                    if (i >= mrows) break;
                    O[(int64_t)i * ld + j] = E[rr * 33 + lane];
                }
            } else if (j < ncols) {
                const int tc = tcol0 + j;
                for (int rr = 0; rr < 32; rr++) {
                    const int i = warp * 32 + rr;
                    if (i >= mrows) break;
                    const int tr = trow_s[i];
                    if (tr < 0) continue;
                    if (lower_only && tr < wf && tc > tr) continue;
                    atomicAdd(&C[(int64_t)tr * ldf + tc], -E[rr * 33 + lane]);
                }
            }
            __syncwarp();
        }
    } else if (tid == 0) {
        atomicAdd(&st->timeout, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
    }
    if (prof && tid == 0) {
        prof[2 * blockIdx.x] = (int64_t)t_start;
        prof[2 * blockIdx.x + 1] = (int64_t)global_ns();
    }
}

}  // namespace pgpu

namespace pgpu {

// ---------------------------------------------------------------------------
// Persistent, warp-specialized form of the same update GEMM: one CTA per SM
// walks the level's tiles (tile = blockIdx.x + i * gridDim.x) with three
// roles running concurrently, so the loads of tile i+1, its MMAs and the
// scatter-add epilogue of tile i overlap:
//   warps 0-3 (128 threads): epilogue -- warp w reads TMEM lanes 32w..32w+31
//                            of the finished accumulator, transposes through
//                            shared memory and scatter-adds into the target;
//   warps 4-11 (2 x 128):    producers -- global -> registers -> (3xTF32:
//                            hi/lo split) -> SWIZZLE_128B shared-memory ring of
//                            TCP_STAGES stages, then mbarrier arrive (full);
//                            the two groups take alternate k-blocks, so two
//                            stages' loads are in flight at once;
//   warp 12, lane 0:         MMA issuer -- waits for a full stage, issues the
//                            tcgen05.mma of the k-block into one of two TMEM
//                            accumulators (2 x 128 columns), commits the stage
//                            back to the producers (empty) and the finished
//                            tile to the epilogue (acc_full); the epilogue
//                            hands the accumulator back (acc_empty).
// Every wait is bounded (mbar_wait): on time-out a role stops, records
// Status::timeout, and the others run out on their own bounded waits; TMEM is
// freed after all roles met at the final barrier.
// ---------------------------------------------------------------------------
constexpr int TCP_PGROUPS = 2;                              // producer groups of 4 warps
constexpr int TCP_MMA_WARP = 4 + 4 * TCP_PGROUPS;
constexpr int TCP_THREADS = 32 * (TCP_MMA_WARP + 1);
template <bool SPLIT> struct TcpCfg;
template <> struct TcpCfg<false> { static constexpr int STAGES = 6, TILES = 2; };
template <> struct TcpCfg<true> { static constexpr int STAGES = 3, TILES = 4; };
constexpr int TCP_EPI_BYTES = 4 * 32 * 33 * 4;
template <bool SPLIT>
constexpr int tcp_smem_bytes() {
    return TcpCfg<SPLIT>::STAGES * TcpCfg<SPLIT>::TILES * TC_TILE_BYTES + TCP_EPI_BYTES + 1024;
}
constexpr int TCP_TMEM_COLS = 256;

// Atomic add of 4 consecutive floats (16-byte aligned address).
__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d) {
    asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}


struct TcTileView {
    const float *A, *B;
    int mrows, ncols, K, nk, flags, c, b, f, arow, j0, i0, M, pair;
    int64_t out;
};

__device__ __forceinline__ TcTileView tc_tile_view(const Meta &m, const int4 tl, const GemmTask *tasks,
                                                   const float *coefL, const float *coefU, const float *inv) {
    const GemmTask t = tasks[tl.x];
    TcTileView v;
    v.c = t.c;
    v.b = t.b;
    v.f = t.f;
    v.flags = t.flags;
    v.out = t.out;
    v.K = m.width[t.c];
    const int ld = m.ld[t.c];
    const bool trsm = (t.flags & 64) != 0;
    const int N = trsm ? v.K : m.blrow[t.b] - m.bfrow[t.b] + 1;
    const int i0 = tl.y * TC_BM;
    v.i0 = i0;
    v.j0 = tl.z * TC_BN;
    v.arow = t.arow0 + i0;
    v.A = ((t.flags & 1) ? coefU : coefL) + m.coefoff[t.c] + (int64_t)(t.arow0 + i0) * ld;
    v.B = trsm ? inv + m.invoff[t.c] + ((t.flags & 128) ? inv_span(v.K, ld) : 0) + (int64_t)v.j0 * ld
               : ((t.flags & 2) ? coefU : coefL) + m.coefoff[t.c] + (int64_t)(m.browoff[t.b] + v.j0) * ld;
    v.mrows = min(TC_BM, t.M - i0);
    v.ncols = min(TC_BN, N - v.j0);
    v.nk = (v.K + TC_BK - 1) / TC_BK;
    v.M = t.M;
    v.pair = tl.w & 1;   // (TMA kernel) rows i0 .. i0 + 255: this tile and the next one of the task
    return v;
}

template <bool SPLIT>
__global__ void __launch_bounds__(TCP_THREADS, 1)
    k_gemm_scatter_tc_persistent(Meta m, const int4 *__restrict__ tiles, int ntiles,
                                 const GemmTask *__restrict__ tasks, float *__restrict__ coefL,
                                 float *__restrict__ coefU, Status *st, const float *__restrict__ inv,
                                 float *__restrict__ scr) {
    constexpr int S = TcpCfg<SPLIT>::STAGES, NT = TcpCfg<SPLIT>::TILES;
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t full[S], empty[S], accf[2], acce[2], drained;
    __shared__ uint32_t tmem_base_s;
    __shared__ int fail_s;
    __shared__ int trow_s[TC_BM];

    const uint32_t raw = smem_u32(tc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char *sbase = tc_smem_raw + (base - raw);
    float *epi = reinterpret_cast<float *>(sbase + S * NT * TC_TILE_BYTES);   // [4][32][33]

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == TCP_MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(TCP_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(smem_u32(&full[s]), 128);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&accf[b]), 1);
            mbar_init(smem_u32(&acce[b]), 128);
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

    if (warp >= 4 && warp < TCP_MMA_WARP) {
        // ---------------- producers ----------------
        // group g fills the k-blocks it with it % TCP_PGROUPS == g, so that
        // the loads of consecutive stages are in flight together
        const int grp = (warp - 4) >> 2;
        const int ptid = tid - 128 * (1 + grp);
        constexpr int CH = (TC_BM * 8) / 128;          // 8 chunks of 16 B per operand per thread
        int it = 0;
        for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x) {
            const TcTileView v = tc_tile_view(m, tiles[ti], tasks, coefL, coefU, inv);
            const int ld = m.ld[v.c];
            for (int kb = 0; kb < v.nk; kb++, it++) {
                if (it % TCP_PGROUPS != grp) continue;
                const int s = it % S;
                const int k0 = kb * TC_BK;
                float4 ra[CH], rb[CH];
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const int e = ptid + q * 128;
                    const int r = e >> 3, kc = k0 + (e & 7) * 4;
                    ra[q] = ((r < v.mrows) && (kc < v.K))
                                ? __ldg(reinterpret_cast<const float4 *>(v.A + (int64_t)r * ld + kc))
                                : make_float4(0.f, 0.f, 0.f, 0.f);
                    rb[q] = ((r < v.ncols) && (kc < v.K))
                                ? __ldg(reinterpret_cast<const float4 *>(v.B + (int64_t)r * ld + kc))
                                : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                const int nmma = tc_mma_n(v.ncols);   // B rows the MMAs read
                if (it >= S && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((it / S - 1) & 1))) {
                    atomicExch(&fail_s, 1);
                    break;
                }
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const int e = ptid + q * 128;
                    const int r = e >> 3, ch = e & 7;
                    const uint32_t soff = (uint32_t)(r * 128 + ((ch ^ (r & 7)) << 4));
                    if (SPLIT) {
                        float4 h, l;
                        h.x = tf32_hi(ra[q].x); h.y = tf32_hi(ra[q].y); h.z = tf32_hi(ra[q].z); h.w = tf32_hi(ra[q].w);
                        l.x = ra[q].x - h.x; l.y = ra[q].y - h.y; l.z = ra[q].z - h.z; l.w = ra[q].w - h.w;
                        sts128(tile_addr(s, 0) + soff, h);
                        sts128(tile_addr(s, 1) + soff, l);
                        if (r < nmma) {
                            h.x = tf32_hi(rb[q].x); h.y = tf32_hi(rb[q].y); h.z = tf32_hi(rb[q].z); h.w = tf32_hi(rb[q].w);
                            l.x = rb[q].x - h.x; l.y = rb[q].y - h.y; l.z = rb[q].z - h.z; l.w = rb[q].w - h.w;
                            sts128(tile_addr(s, 2) + soff, h);
                            sts128(tile_addr(s, 3) + soff, l);
                        }
                    } else {
                        sts128(tile_addr(s, 0) + soff, ra[q]);
                        if (r < nmma) sts128(tile_addr(s, 1) + soff, rb[q]);
                    }
                }
                tc_fence_async_smem();
                mbar_arrive(smem_u32(&full[s]));
            }
        }
    } else if (warp == TCP_MMA_WARP) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int it = 0, tl = 0;
            for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x, tl++) {
                const TcTileView v = tc_tile_view(m, tiles[ti], tasks, coefL, coefU, inv);
                const uint32_t idesc = tc_idesc(tc_mma_n(v.ncols));
                const int ab = tl & 1;
                const uint32_t acc = tmem + (uint32_t)(ab * 128);
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
                            const uint64_t ah = tc_sdesc(tile_addr(s, 0) + kk * 32),
                                           al = tc_sdesc(tile_addr(s, 1) + kk * 32);
                            const uint64_t bh = tc_sdesc(tile_addr(s, 2) + kk * 32),
                                           bl = tc_sdesc(tile_addr(s, 3) + kk * 32);
                            tc_mma(acc, al, bh, idesc, first);
                            tc_mma(acc, ah, bl, idesc, 1u);
                            tc_mma(acc, ah, bh, idesc, 1u);
                        } else {
                            tc_mma(acc, tc_sdesc(tile_addr(s, 0) + kk * 32), tc_sdesc(tile_addr(s, 1) + kk * 32),
                                   idesc, first);
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
            // every MMA this thread issued has completed before TMEM is freed
            tc_commit(smem_u32(&drained));
            if (!mbar_wait(smem_u32(&drained), 0u)) atomicExch(&fail_s, 1);
        }
    } else {
        // ---------------- epilogue (warps 0-3) ----------------
        float *E = epi + warp * 32 * 33;
        int tl = 0;
        for (int ti = blockIdx.x; ti < ntiles && !failed(); ti += gridDim.x, tl++) {
            const TcTileView v = tc_tile_view(m, tiles[ti], tasks, coefL, coefU, inv);
            const int ab = tl & 1;
            // target panel row of my accumulator row (binary search in f's blocks)
            const int myrow = warp * 32 + lane;
            const bool trsm = (v.flags & 64) != 0;
            int tr = -1;
            if (myrow < v.mrows && !trsm) tr = panel_row_of(m, v.f, m.rowidx[m.rowbase[v.c] + v.arow + myrow]);
            if (!mbar_wait(smem_u32(&accf[ab]), (uint32_t)((tl / 2) & 1))) {
                atomicExch(&fail_s, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            trow_s[myrow] = tr;
            __syncwarp();
            float *C = ((v.flags & 4) ? coefU : coefL) + m.coefoff[v.f];
            const int ldf = m.ld[v.f], wf = m.width[v.f];
            const int tcol0 = m.bfrow[v.b] + v.j0 - m.fcol[v.f];
            const bool lower_only = (v.flags & 8) != 0;
            for (int cb = 0; cb < TC_BN; cb += 32) {
                uint32_t r[32];
                tc_ld32(tmem + (uint32_t)(ab * 128) + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, r);
                __syncwarp();
#pragma unroll
                for (int q = 0; q < 32; q++) E[lane * 33 + q] = __uint_as_float(r[q]);
                __syncwarp();
                const int j = cb + lane;
                if (j < v.ncols && trsm) {
                    const int ldc = m.ld[v.c];
                    float *O = scr + v.out + (int64_t)v.i0 * ldc + v.j0;
                    for (int rr = 0; rr < 32; rr++) {
                        const int i = warp * 32 + rr;
                        if (i >= v.mrows) break;
                        O[(int64_t)i * ldc + j] = E[rr * 33 + lane];
                    }
                } else if (!trsm && cb < v.ncols) {
                    // scatter-add with 16-byte vector reductions: the block's
                    // target columns [tcs, tcs + nvalid) lie in 9 groups of 4
                    // columns aligned in the target row (any alignment of
                    // tcs); entries outside it, or masked, add zero
                    const int nvalid = min(32, v.ncols - cb);
                    const int tcs = tcol0 + cb, a0 = tcs & ~3, o = tcs - a0;
                    for (int k = lane; k < 32 * 9; k += 32) {
                        const int rr = k / 9, g = k - rr * 9;
                        const int t2 = trow_s[warp * 32 + rr];     // -1: no target (or row past the tile)
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
            mbar_arrive(smem_u32(&acce[ab]));
        }
    }
    if (tid == 0 && failed()) atomicAdd(&st->timeout, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == TCP_MMA_WARP) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCP_TMEM_COLS)
                     : "memory");
    }
}

}  // namespace pgpu
