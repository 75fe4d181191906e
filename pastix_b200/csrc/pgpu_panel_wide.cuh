// Diagonal-block factorization of wide cblks (w of a few hundred columns, the
// separators near the root of the elimination tree, whose off-diagonal rows
// are solved afterwards by the inverse + GEMM path): the same factorization
// as k_panel_factor with rows = w (kernels/core_zpotrfsp.c:144
// core_zpotrfsp, kernels/core_zgetrfsp.c:138 core_zgetrfsp,
// kernels/core_zsytrfsp.c:141 / core_zhetrfsp.c:144), reorganized for one
// 512-thread CTA per cblk as a left-looking (Crout) sweep over column blocks
// of PB = 32:
//
//   for each column block jb:
//     1. C = A[jb:w, jb:jb+nb] (and for LU R = A[jb:jb+nb, jb+nb:w]^t) is
//        copied to shared memory (cp.async, in flight during step 2);
//     2. C -= L[jb:w, 0:jb] op(L[jb:jb+nb, 0:jb] D)^t       (LL^h, LDL^t/h)
//        C -= L[jb:w, 0:jb] U[0:jb, jb:jb+nb]               (LU, L side)
//        R -= U[0:jb, jb+nb:w]^t L[jb:jb+nb, 0:jb]^t        (LU, U side)
//        with the finished columns streamed through shared memory in
//        chunks of kc columns (double-buffered cp.async), 4 x 4 register
//        tiles per thread (rows strided by the row-group count, columns by
//        8, so that each warp's 16-byte loads hit distinct banks);
//     3. one warp factorizes the nb x nb tile (static pivoting), the rows
//        below are solved against it one thread per row (LU: and the
//        columns of R against its unit lower part);
//     4. C (and R) are written back.
//
// Compared with the right-looking k_panel_factor the trailing matrix is
// never re-read and re-written through L2 for every column block: each
// finished column block is read once per later block as a chunk operand.
#pragma once

#include "pgpu_common.cuh"
#include "pgpu_panel.cuh"

namespace pgpu {

constexpr int WP_THREADS = 512, WP_WARPS = WP_THREADS / 32;

// Tiles a thread owns: C tiles (rows of the block column) plus, for LU, R
// tiles (columns of the row block); 4 x 4 entries each.
template <int MODE>
constexpr int wp_ntt() { return MODE == FM_GETRF ? 3 : 2; }

// Row groups of a tile set over m rows: ceil(m / 4) rounded up to a multiple
// of 4, so that every warp's 32 tiles are of one kind.
__host__ __device__ inline int wp_row_groups(int m) { return (((m + 3) >> 2) + 3) & ~3; }

template <typename T>
__device__ __forceinline__ void wp_lds16(const T *p, T (&v)[16 / sizeof(T)]) {
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    memcpy(v, &u, 16);
}

// Row solve against the factorized tile with the row in registers (fully
// unrolled, so x stays out of local memory):
//   x[j] = (x[j] - sum_{l<j} x[l] op(C[j][l])) * (UNIT ? 1 : rdiag[j])
// in increasing l, C row-major with 16-byte rows (ldc), read as broadcast
// vectors.  C = the tile's lower part (LL^h, LDL rows; LU row block, unit),
// or the transposed upper part (LU rows: x U = a).
template <typename T, bool CJ, bool UNIT>
__device__ __forceinline__ void wp_solve_rows(T (&x)[PB], const T *C, int ldc, const T *rdiag, int nb) {
    constexpr int VK = 16 / sizeof(T);
#pragma unroll
    for (int j = 0; j < PB; j++)
        if (j < nb) {
            T s = x[j];
#pragma unroll
            for (int l0 = 0; l0 < j; l0 += VK) {
                T c[VK];
                wp_lds16<T>(C + j * ldc + l0, c);
#pragma unroll
                for (int v = 0; v < VK; v++)
                    if (l0 + v < j) s -= x[l0 + v] * cj<CJ>(c[v]);
            }
            x[j] = UNIT ? s : s * rdiag[j];
        }
}

// Byte offset of the tile operands TA / TB, and the shared memory of
// k_panel_wide for width w with chunks of kcb bytes per row.
__host__ __device__ inline size_t wp_tile_offset(int w, size_t esz, bool lu, bool ldl, int kcb) {
    const size_t chunk_row = (size_t)kcb + 16;
    const size_t b = 2 * (size_t)(w + 16) * chunk_row * (lu ? 2 : 1) + (size_t)w * PBL * esz * (lu ? 2 : 1) +
                     (ldl ? (size_t)w * esz : 0);
    return (b + 15) / 16 * 16;
}
__host__ inline size_t wp_smem_bytes(int w, size_t esz, bool lu, bool ldl, int kcb) {
    return wp_tile_offset(w, esz, lu, ldl, kcb) + (size_t)(lu ? 2 : 1) * PB * (PB * esz + 16);
}

// The register tile factorization as a call of its own: the kernel's live
// state is saved around the call, so the fully unrolled factorization gets
// the register file to itself (inlined, it competes with the 512-thread
// budget and runs about 1.5x slower).
template <typename T, int MODE>
__device__ __noinline__ void wp_factor_tile_call(T *Cb, int nb, typename real_of<T>::type crit, int *npiv, int *nneg,
                                                 int *nbad) {
    int a = 0, b = 0, c = 0;
    warp_factor_tile<T, MODE>(Cb, nb, crit, a, b, c);
    *npiv += a;
    *nneg += b;
    *nbad += c;
}

// Shared memory (elements of T): Ach[2][w + 16][kc + VK] chunk buffers of
// the left columns, for LU Uch[2][w + 16][kc + VK] (the U rows above,
// transposed), C[w][PBL], for LU R[w][PBL], for LDL d[w], then (16-byte
// aligned) the factorized tile as row solve operands TA[PB][PB + VK] and
// for LU TB[PB][PB + VK].
template <typename T, int MODE>
__global__ void __launch_bounds__(WP_THREADS) k_panel_wide(Meta m, const int2 *__restrict__ jobs,
                                                           T *__restrict__ coefL, const double *critp, int kc,
                                                           Status *st, int64_t *prof) {
    typedef typename real_of<T>::type R;
    constexpr bool LU = (MODE == FM_GETRF);
    constexpr bool LDL = fm_ldl(MODE);
    constexpr bool CJ = fm_conj(MODE);
    constexpr int VK = 16 / sizeof(T);
    constexpr int NTT = wp_ntt<MODE>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T rdiag[PB];                        // 1 / op(tile diagonal); LDL: 1 / d
    const int2 job = jobs[blockIdx.x];
    const int c = job.x;
    const int w = m.width[c], ld = m.ld[c];
    T *A = coefL + m.coefoff[c];
    const int S = kc + VK;                         // chunk row stride: 16 bytes of padding
    const int64_t bufsz = (int64_t)(w + 16) * S;   // w rows + the tiles' overhang
    T *Ach = reinterpret_cast<T *>(smem_raw);
    T *Uch = Ach + 2 * bufsz;                      // buffer b of Uch = Ach + (2 + b) * bufsz
    T *Cb = Uch + (LU ? 2 * bufsz : 0);
    T *Rb = Cb + (int64_t)w * PBL;
    T *dsm = Rb + (LU ? (int64_t)w * PBL : 0);
    constexpr int LDT = PB + VK;
    T *TA = reinterpret_cast<T *>(smem_raw + wp_tile_offset(w, sizeof(T), LU, LDL, kc * (int)sizeof(T)));
    T *TB = TA + PB * LDT;
    const R crit = R(*critp);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t t_start = prof ? global_ns() : 0;
    int npiv = 0, nneg = 0, nbad = 0;

    for (int jb = 0; jb < w; jb += PB) {
        const int nb = min(PB, w - jb), M = w - jb, MR = LU ? M - nb : 0;
        // 1. the block column (and the row block right of the tile), in flight during the update
        // (warp = row, lane = column: no index divisions)
        if (lane < nb)
            for (int r = warp; r < M; r += WP_WARPS)
                cp_async_ca<sizeof(T)>(smem_u32(Cb + r * PBL + lane), A + (int64_t)(jb + r) * ld + jb + lane);
        if constexpr (LU)
            for (int j = warp; j < nb; j += WP_WARPS)
                for (int i = lane; i < MR; i += 32)
                    cp_async_ca<sizeof(T)>(smem_u32(Rb + i * PBL + j), A + (int64_t)(jb + j) * ld + jb + nb + i);
        cp_async_commit();
        // 2. left-looking update with the finished columns [0, jb)
        const int RG = wp_row_groups(M), RG2 = LU ? wp_row_groups(MR) : 0;
        const int ntiles = (RG + RG2) * 8;
        T acc[NTT][4][4];
        if (jb > 0) {
            auto stage = [&](int bf, int k0) {
                T *dA = Ach + bf * bufsz;
                const int lp = __ffs(kc / VK) - 1;   // 16-byte pieces per row: a power of two
                for (int e = tid; e < (M << lp); e += WP_THREADS) {
                    const int r = e >> lp, pc = e - (r << lp);
                    cp_async16(smem_u32(dA + r * S + pc * VK), A + (int64_t)(jb + r) * ld + k0 + pc * VK, true);
                }
                if (LU) {
                    T *dU = Uch + bf * bufsz;
                    for (int kk = warp; kk < kc; kk += WP_WARPS)
                        for (int i = lane; i < M; i += 32)
                            cp_async_ca<sizeof(T)>(smem_u32(dU + i * S + kk), A + (int64_t)(k0 + kk) * ld + jb + i);
                }
            };
            // operand rows of each owned tile, as element offsets from Ach
            // (buffer 0): left row p at lo[t] + p * ls[t], right row q at
            // ro[t] + 8 q S.  Rows past the valid ones (up to M + 15) stay
            // inside the buffers and only feed entries that are discarded.
            int lo[NTT], ls[NTT], ro[NTT];
#pragma unroll
            for (int t = 0; t < NTT; t++) {
                const int u = tid + t * WP_THREADS;
                const bool rt = LU && u >= RG * 8;     // an R tile
                const int uu = rt ? u - RG * 8 : u;
                const int ti = uu >> 3, tj = uu & 7;
                // C tile: left = L rows (Ach), right = L rows (Ach) or U^t rows (Uch)
                // R tile: left = U^t rows nb.. (Uch), right = L rows (Ach)
                lo[t] = rt ? (int)(2 * bufsz) + (nb + ti) * S : ti * S;
                ls[t] = (rt ? RG2 : RG) * S;
                ro[t] = (LU && !rt) ? (int)(2 * bufsz) + tj * S : tj * S;
#pragma unroll
                for (int p = 0; p < 4; p++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[t][p][q] = T(0);
            }
            const int nck = jb / kc;
            stage(0, 0);
            cp_async_commit();
            for (int ck = 0; ck < nck; ck++) {
                if (ck + 1 < nck) stage((ck + 1) & 1, (ck + 1) * kc);
                cp_async_commit();
                cp_async_wait<1>();
                __syncthreads();
                const T *base = Ach + (ck & 1) * bufsz;
                const int k0 = ck * kc;
#pragma unroll
                for (int t = 0; t < NTT; t++) {
                    if (tid + t * WP_THREADS >= ntiles) break;     // whole warps (ntiles is a multiple of 32)
#pragma unroll 2
                    for (int kk = 0; kk < kc; kk += VK) {
                        T a[4][VK], b[4][VK];
#pragma unroll
                        for (int p = 0; p < 4; p++) wp_lds16<T>(base + lo[t] + p * ls[t] + kk, a[p]);
#pragma unroll
                        for (int q = 0; q < 4; q++) wp_lds16<T>(base + ro[t] + q * 8 * S + kk, b[q]);
#pragma unroll
                        for (int v = 0; v < VK; v++) {
                            T dk = T(1);
                            if (LDL) dk = dsm[k0 + kk + v];
#pragma unroll
                            for (int q = 0; q < 4; q++) {
                                T bq = cj<CJ>(b[q][v]);
                                if (LDL) bq = bq * dk;
#pragma unroll
                                for (int p = 0; p < 4; p++) acc[t][p][q] += a[p][v] * bq;
                            }
                        }
                    }
                }
                __syncthreads();                  // the buffer is refilled two chunks later
            }
        }
        cp_async_wait<0>();
        __syncthreads();
        if (jb > 0) {
#pragma unroll
            for (int t = 0; t < NTT; t++) {
                const int u = tid + t * WP_THREADS;
                if (u >= ntiles) break;
                const bool rt = u >= RG * 8;
                const int uu = rt ? u - RG * 8 : u;
                const int ti = uu >> 3, tj = uu & 7;
                const int rg = rt ? RG2 : RG, rows = rt ? MR : M;
                T *D = rt ? Rb : Cb;
#pragma unroll
                for (int p = 0; p < 4; p++) {
                    const int r = ti + p * rg;
                    if (r >= rows) continue;
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int j = tj + 8 * q;
                        if (j < nb) D[r * PBL + j] -= acc[t][p][q];
                    }
                }
            }
            __syncthreads();
        }
        // 3. the tile, then the rows below it (and the columns of R)
        if (tid < 32) {
            if constexpr (sizeof(T) == 4) wp_factor_tile_call<T, MODE>(Cb, nb, crit, &npiv, &nneg, &nbad);
            else warp_factor_tile_smem<T, MODE>(Cb, nb, crit, npiv, nneg, nbad);
            if (tid < nb) {
                const T d = Cb[tid * PBL + tid];
                if (LDL) dsm[jb + tid] = d;
                rdiag[tid] = T(1) / (MODE == FM_POTRF ? cj<CJ>(d) : d);
            }
            // the tile as 16-byte rows: TA = lower part (LU: U^t), TB = lower part (LU)
            if (tid < nb)
                for (int j = 0; j < nb; j++) {
                    const int l = tid;
                    TA[j * LDT + l] = LU ? Cb[l * PBL + j] : Cb[j * PBL + l];
                    if (LU) TB[j * LDT + l] = Cb[j * PBL + l];
                }
        }
        __syncthreads();
        for (int r = nb + tid; r < M; r += WP_THREADS) {
            T x[PB];
#pragma unroll
            for (int j = 0; j < PB; j++) x[j] = (j < nb) ? Cb[r * PBL + j] : T(0);
            if (LU) wp_solve_rows<T, false, false>(x, TA, LDT, rdiag, nb);
            else if (LDL) wp_solve_rows<T, CJ, true>(x, TA, LDT, rdiag, nb);
            else wp_solve_rows<T, CJ, false>(x, TA, LDT, rdiag, nb);
#pragma unroll
            for (int j = 0; j < PB; j++)
                if (j < nb) Cb[r * PBL + j] = LDL ? x[j] * rdiag[j] : x[j];
        }
        if constexpr (LU)
            for (int i = tid; i < MR; i += WP_THREADS) {
                T y[PB];
#pragma unroll
                for (int j = 0; j < PB; j++) y[j] = (j < nb) ? Rb[i * PBL + j] : T(0);
                wp_solve_rows<T, false, true>(y, TB, LDT, rdiag, nb);
#pragma unroll
                for (int j = 0; j < PB; j++)
                    if (j < nb) Rb[i * PBL + j] = y[j];
            }
        __syncthreads();
        // 4. write back (the symmetric forms keep the tile's lower triangle only)
        if (lane < nb)
            for (int r = warp; r < M; r += WP_WARPS)
                if (LU || r >= nb || lane <= r) A[(int64_t)(jb + r) * ld + jb + lane] = Cb[r * PBL + lane];
        if constexpr (LU)
            for (int j = warp; j < nb; j += WP_WARPS)
                for (int i = lane; i < MR; i += 32) A[(int64_t)(jb + j) * ld + jb + nb + i] = Rb[i * PBL + j];
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
// Lookahead form for single-precision LL^t / LDL^t (the 100^3 root chain's
// case): while warp 0 factorizes the tile of block column jb, warps 1-15
// already update block column jb + 32 with the finished columns [0, jb)
// (chunks from global memory, a named barrier among those 480 threads);
// after the row solves of block jb the last contribution, columns
// [jb, jb + 32), comes from the just-solved block column, staged once in
// the chunk layout (the "tail").  The same products as k_panel_wide, the
// sums for an entry taken in the same chunk order.
// Shared memory (floats): Ach[2][w + 16][36], C[2][w][PBL] (this block
// column and the next), d[w] (LDL), TA[PB][36].
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t wpla_tile_offset(int w, bool ldl) {
    const size_t b = (2 * (size_t)(w + 16) * 36 + 2 * (size_t)w * PBL + (ldl ? (size_t)w : 0)) * sizeof(float);
    return (b + 15) / 16 * 16;
}
__host__ inline size_t wpla_smem_bytes(int w, bool ldl) { return wpla_tile_offset(w, ldl) + (size_t)PB * 36 * 4; }

__device__ __forceinline__ void wpla_bar_rest() { asm volatile("bar.sync 1, %0;" ::"n"(WP_THREADS - 32) : "memory"); }

template <int MODE>
__global__ void __launch_bounds__(WP_THREADS) k_panel_wide_la(Meta m, const int2 *__restrict__ jobs,
                                                              float *__restrict__ coefL, const double *critp,
                                                              Status *st, int64_t *prof) {
    typedef float T;
    constexpr bool LDL = fm_ldl(MODE);
    constexpr int VK = 4, KC = 32, S = KC + VK, NTT = 2, GT = WP_THREADS - 32, LDT = PB + VK;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T rdiag[PB];
    const int2 job = jobs[blockIdx.x];
    const int c = job.x;
    const int w = m.width[c], ld = m.ld[c];
    T *A = coefL + m.coefoff[c];
    const int bufsz = (w + 16) * S;
    T *Ach = reinterpret_cast<T *>(smem_raw);
    T *Cbuf = Ach + 2 * bufsz;                         // C[2][w][PBL]
    T *dsm = Cbuf + 2 * w * PBL;
    T *TA = reinterpret_cast<T *>(smem_raw + wpla_tile_offset(w, LDL));
    const T crit = T(*critp);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t t_start = prof ? global_ns() : 0;
    int npiv = 0, nneg = 0, nbad = 0;

    // acc[t] += left rows (lo[t] + p ls) x right rows (ro[t] + 8 q S) over one chunk
    auto chunk_fma = [&](const T *base, const int (&lo)[NTT], int ls, const int (&ro)[NTT], int tbase, int nthr,
                         int ntiles, int k0, T (&acc)[NTT][4][4]) {
#pragma unroll
        for (int t = 0; t < NTT; t++) {
            if (tbase + t * nthr >= ntiles) break;     // whole warps
#pragma unroll 2
            for (int kk = 0; kk < KC; kk += VK) {
                T a[4][VK], b[4][VK];
#pragma unroll
                for (int p = 0; p < 4; p++) wp_lds16<T>(base + lo[t] + p * ls + kk, a[p]);
#pragma unroll
                for (int q = 0; q < 4; q++) wp_lds16<T>(base + ro[t] + q * 8 * S + kk, b[q]);
#pragma unroll
                for (int v = 0; v < VK; v++) {
                    T dk = T(1);
                    if (LDL) dk = dsm[k0 + kk + v];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const T bq = LDL ? b[q][v] * dk : b[q][v];
#pragma unroll
                        for (int p = 0; p < 4; p++) acc[t][p][q] += a[p][v] * bq;
                    }
                }
            }
        }
    };
    // tiles of thread tbase over mrows x 32: operand rows and zeroed accumulators
    auto tiles_setup = [&](int tbase, int nthr, int rg, int (&lo)[NTT], int (&ro)[NTT], T (&acc)[NTT][4][4]) {
#pragma unroll
        for (int t = 0; t < NTT; t++) {
            const int u = tbase + t * nthr;
            lo[t] = (u >> 3) * S;
            ro[t] = (u & 7) * S;
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[t][p][q] = T(0);
        }
    };
    auto tiles_subtract = [&](T *D, int tbase, int nthr, int rg, int ntiles, int rows, int nbc, T (&acc)[NTT][4][4]) {
#pragma unroll
        for (int t = 0; t < NTT; t++) {
            const int u = tbase + t * nthr;
            if (u >= ntiles) break;
            const int ti = u >> 3, tj = u & 7;
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const int r = ti + p * rg;
                if (r >= rows) continue;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int j = tj + 8 * q;
                    if (j < nbc) D[r * PBL + j] -= acc[t][p][q];
                }
            }
        }
    };

    // block column 0
    {
        const int nb0 = min(PB, w);
        if (lane < nb0)
            for (int r = warp; r < w; r += WP_WARPS)
                cp_async_ca<4>(smem_u32(Cbuf + r * PBL + lane), A + (int64_t)r * ld + lane);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
    }
    int cur = 0;
    for (int jb = 0; jb < w; jb += PB) {
        const int nb = min(PB, w - jb), M = w - jb;
        T *Cc = Cbuf + cur * w * PBL, *Cn = Cbuf + (cur ^ 1) * w * PBL;
        const int jn = jb + PB, Mn = w - jn, nbn = min(PB, w - jn);
        const bool has_next = jn < w;
        const int RGn = has_next ? wp_row_groups(Mn) : 0, ntn = RGn * 8;
        if (warp == 0) {
            // 1a. the tile of block jb
            wp_factor_tile_call<T, MODE>(Cc, nb, crit, &npiv, &nneg, &nbad);
            if (lane < nb) {
                const T d = Cc[lane * PBL + lane];
                if (LDL) dsm[jb + lane] = d;
                rdiag[lane] = T(1) / d;
                for (int j = 0; j < nb; j++) TA[j * LDT + lane] = Cc[j * PBL + lane];
            }
        } else if (has_next) {
            // 1b. (warps 1-15) block column jn: load, and its update with the columns [0, jb)
            const int gt = tid - 32, gw = warp - 1;
            if (lane < nbn)
                for (int r = gw; r < Mn; r += WP_WARPS - 1)
                    cp_async_ca<4>(smem_u32(Cn + r * PBL + lane), A + (int64_t)(jn + r) * ld + jn + lane);
            cp_async_commit();
            if (jb > 0) {
                int lo[NTT], ro[NTT];
                T acc[NTT][4][4];
                tiles_setup(gt, GT, RGn, lo, ro, acc);
                auto stage = [&](int bf, int k0) {
                    T *dA = Ach + bf * bufsz;
                    for (int e = gt; e < (Mn << 3); e += GT) {
                        const int r = e >> 3, pc = e & 7;
                        cp_async16(smem_u32(dA + r * S + pc * VK), A + (int64_t)(jn + r) * ld + k0 + pc * VK, true);
                    }
                };
                const int nck = jb / KC;
                stage(0, 0);
                cp_async_commit();
                for (int ck = 0; ck < nck; ck++) {
                    if (ck + 1 < nck) stage((ck + 1) & 1, (ck + 1) * KC);
                    cp_async_commit();
                    cp_async_wait<1>();
                    wpla_bar_rest();
                    chunk_fma(Ach + (ck & 1) * bufsz, lo, RGn * S, ro, gt, GT, ntn, ck * KC, acc);
                    wpla_bar_rest();
                }
                cp_async_wait<0>();
                wpla_bar_rest();
                tiles_subtract(Cn, gt, GT, RGn, ntn, Mn, nbn, acc);
            } else {
                cp_async_wait<0>();
            }
        }
        __syncthreads();
        // 2. the rows below the tile
        for (int r = nb + tid; r < M; r += WP_THREADS) {
            T x[PB];
#pragma unroll
            for (int j = 0; j < PB; j++) x[j] = (j < nb) ? Cc[r * PBL + j] : T(0);
            if (LDL) wp_solve_rows<T, false, true>(x, TA, LDT, rdiag, nb);
            else wp_solve_rows<T, false, false>(x, TA, LDT, rdiag, nb);
#pragma unroll
            for (int j = 0; j < PB; j++)
                if (j < nb) Cc[r * PBL + j] = LDL ? x[j] * rdiag[j] : x[j];
        }
        __syncthreads();
        // 3. write back; the solved rows below the tile, staged as the tail chunk of block jn
        if (lane < nb)
            for (int r = warp; r < M; r += WP_WARPS) {
                const T v = Cc[r * PBL + lane];
                if (r >= nb || lane <= r) A[(int64_t)(jb + r) * ld + jb + lane] = v;
                if (has_next && r >= PB) Ach[(r - PB) * S + lane] = v;
            }
        __syncthreads();
        // 4. the tail: block jn -= (rows jn.. of block jb) op(rows jn..jn+32 of block jb D)^t
        if (has_next) {
            int lo[NTT], ro[NTT];
            T acc[NTT][4][4];
            tiles_setup(tid, WP_THREADS, RGn, lo, ro, acc);
            chunk_fma(Ach, lo, RGn * S, ro, tid, WP_THREADS, ntn, jb, acc);
            tiles_subtract(Cn, tid, WP_THREADS, RGn, ntn, Mn, nbn, acc);
        }
        __syncthreads();
        cur ^= 1;
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
// Cblks of at most 32 columns (the leaves, ~10^5-10^6 of them in the
// batched 2D problems): one warp per cblk.  The w x w diagonal block is one
// tile, factorized by the warp in shared memory (warp_factor_tile_smem: with
// every warp of the SM in it, the fully unrolled register form misses in the
// instruction cache), and the panel rows below
// it are solved one lane per row with the row in registers -- the same
// operations as k_panel_factor for such a cblk, without a 256-thread CTA per
// leaf.
// Shared memory per warp: X [PB][PB + VK] (the tile with row length PBL
// while it is factorized, then TA, the tile as 16-byte rows for the row
// solves), TB [PB][PB + VK] for LU, 1 / op(diagonal) [PB].
// ---------------------------------------------------------------------------
constexpr int PS_WARPS = 8;
template <typename T>
__host__ __device__ constexpr int ps_warp_elems(bool lu) { return (lu ? 2 : 1) * PB * (PB + 16 / (int)sizeof(T)) + PB; }
template <typename T>
constexpr int ps_smem_bytes(bool lu) { return PS_WARPS * ps_warp_elems<T>(lu) * (int)sizeof(T); }

template <typename T, int MODE>
__global__ void __launch_bounds__(PS_WARPS * 32) k_panel_small(Meta m, const int2 *__restrict__ jobs, int njobs,
                                                               T *__restrict__ coefL, T *__restrict__ coefU,
                                                               const double *critp, int fuse_rows, Status *st) {
    typedef typename real_of<T>::type R;
    constexpr bool LU = (MODE == FM_GETRF);
    constexpr bool LDL = fm_ldl(MODE);
    constexpr bool CJ = fm_conj(MODE);
    constexpr int VK = 16 / sizeof(T), LDT = PB + VK;
    static_assert(LDT >= PBL, "the tile fits in TA");
    extern __shared__ __align__(16) unsigned char ps_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * PS_WARPS + warp;
    if (q >= njobs) return;                        // whole warps; warp-level synchronization only
    T *TA = reinterpret_cast<T *>(ps_raw) + (size_t)warp * ps_warp_elems<T>(LU);
    T *tile = TA;
    T *TB = TA + PB * LDT;
    T *rdiag = TA + (LU ? 2 : 1) * PB * LDT;
    const int c = jobs[q].x;
    const int w = m.width[c], h = m.height[c], ld = m.ld[c];
    const int rows = (h <= fuse_rows) ? h : w;
    T *A = coefL + m.coefoff[c];
    T *AU = coefU + m.coefoff[c];
    const R crit = R(*critp);
    int npiv = 0, nneg = 0, nbad = 0;
    if (lane < w)
        for (int i = 0; i < w; i++) tile[i * PBL + lane] = A[(int64_t)i * ld + lane];
    __syncwarp();
    warp_factor_tile_smem<T, MODE>(tile, w, crit, npiv, nneg, nbad);
    __syncwarp();
    if (lane < w) {
        for (int i = 0; i < w; i++)
            if (LU || lane <= i) A[(int64_t)i * ld + lane] = tile[i * PBL + lane];
        const T d = tile[lane * PBL + lane];
        rdiag[lane] = T(1) / (MODE == FM_POTRF ? cj<CJ>(d) : d);
        if (LU)
            for (int j = 0; j < w; j++) TB[j * LDT + lane] = tile[j * PBL + lane];
    }
    {   // TA over the tile's storage: the whole tile goes through registers
        T v[PB];
#pragma unroll
        for (int j = 0; j < PB; j++)
            v[j] = (lane < w && j < w) ? (LU ? tile[lane * PBL + j] : tile[j * PBL + lane]) : T(0);
        __syncwarp();
#pragma unroll
        for (int j = 0; j < PB; j++)
            if (lane < w && j < w) TA[j * LDT + lane] = v[j];
    }
    __syncwarp();
    for (int r = w + lane; r < rows; r += 32) {
        T x[PB];
        T *row = A + (int64_t)r * ld;
#pragma unroll
        for (int j = 0; j < PB; j++) x[j] = (j < w) ? row[j] : T(0);
        if (LU) wp_solve_rows<T, false, false>(x, TA, LDT, rdiag, w);
        else if (LDL) wp_solve_rows<T, CJ, true>(x, TA, LDT, rdiag, w);
        else wp_solve_rows<T, CJ, false>(x, TA, LDT, rdiag, w);
#pragma unroll
        for (int j = 0; j < PB; j++)
            if (j < w) row[j] = LDL ? x[j] * rdiag[j] : x[j];
        if constexpr (LU) {   // the U^t rows: x L^t = a (unit)
            T *urow = AU + (int64_t)r * ld;
#pragma unroll
            for (int j = 0; j < PB; j++) x[j] = (j < w) ? urow[j] : T(0);
            wp_solve_rows<T, false, true>(x, TB, LDT, rdiag, w);
#pragma unroll
            for (int j = 0; j < PB; j++)
                if (j < w) urow[j] = x[j];
        }
    }
    if (lane == 0) {
        if (npiv) atomicAdd(&st->nbpivots, npiv);
        if (nneg) atomicAdd(&st->negpivots, nneg);
        if (nbad) atomicAdd(&st->nonfinite, nbad);
    }
}

// Whether one CTA covers width w with its tile budget.
__host__ inline bool wp_tiles_fit(int w, bool lu) {
    const int rg = wp_row_groups(w), rg2 = lu ? wp_row_groups(w > PB ? w - PB : 0) : 0;
    return (rg + rg2) * 8 <= (lu ? 3 : 2) * WP_THREADS;
}

}  // namespace pgpu
