// Forward/backward supernodal triangular solves (kernels/solve_ztrsmsp.c) and
// the vector kernels of the iterative refinement (bcsc/bcsc_zspmv.c,
// bcsc/bvec_zcompute.c).  Right-hand sides are column-major n x nrhs in the
// permuted numbering.
#pragma once

#include "pgpu_common.cuh"

namespace pgpu {

constexpr int SOLVE_MAXRHS = 16;

// element count rounded up to a whole number of 16-byte vectors
template <typename T>
__host__ __device__ inline size_t align16_elems(size_t n) {
    const size_t v = 16 / sizeof(T) > 0 ? 16 / sizeof(T) : 1;
    return (n + v - 1) / v * v;
}

// ---------------------------------------------------------------------------
// Forward, diagonal part (kernels/solve_ztrsmsp.c:75 solve_blok_ztrsm with
// Left, Lower, NoTrans): B[fcol:fcol+w, :] := D^{-1} B[...], D = L_kk
// (POTRF, non-unit) or the unit lower part of the LU / LDL diagonal block.
// One CTA per cblk of the level, blocked by 32 columns: warp 0 substitutes
// through the 32x32 tile (shuffles, no block barrier), then all threads
// update the rows below from the tile's column panel, which is first staged
// in shared memory with coalesced loads, pch rows at a time (one round of
// loads per chunk instead of a serial chain of global loads per thread).
// ---------------------------------------------------------------------------
// Diagonal solve of a cblk whose factorization left the inverse of its
// diagonal block (the panel TRSM done as a GEMM): Binv = op(L)^{-1}, each row
// n divided by d_n for LDL.  Forward: y = L^{-1} b, y_n = sum_k
// op(Binv[n][k] s_n) b_k (s_n = d_n for LDL, else 1); backward: x = op(L)^{-t} z,
// x_k = sum_n Binv[n][k] s_n z_n.  The rows of Binv are staged in shared
// memory pch rows at a time (coalesced), the dot products run from there:
// one burst of loads per chunk instead of a chain per 32-column tile.
template <typename T>
__device__ void diag_solve_inverse(const T *__restrict__ Bi, const T *__restrict__ D, int w, int ld, int nrhs,
                                   bool backward, bool ldl, bool cjp, T *__restrict__ v, T *__restrict__ outp,
                                   T *__restrict__ P, int pch, T *__restrict__ Bg, int64_t ldb, int fc) {
    const int tid = threadIdx.x, nt = blockDim.x;
    constexpr int VEC = 16 / sizeof(T);       // elements per 16-byte vector (rows of Bi are 16-byte aligned)
    // v: [w][nrhs] right-hand side in shared memory; outp: [w][nrhs] accumulators (backward)
    if (backward) {
        for (int e = tid; e < w * nrhs; e += nt) outp[e] = T(0);
        if (ldl)   // x_k = sum_n Binv[n][k] (d_n z_n): scale z by D first
            for (int e = tid; e < w * nrhs; e += nt) v[e] = v[e] * D[(int64_t)(e / nrhs) * ld + e / nrhs];
    }
    for (int n0 = 0; n0 < w; n0 += pch) {
        const int nr = min(pch, w - n0), kmax = n0 + nr;     // rows n0..n0+nr, columns 0..kmax
        const int kv = (kmax + VEC - 1) / VEC, kp = kv * VEC;  // 16-byte vectors per row, padded row length
        __syncthreads();
        // rows of Binv are zero beyond the diagonal and in the padding (the
        // workspace is cleared when the plan is built), so whole vectors move
        batched_copy<4>(
            nr * kv, tid, nt,
            [&](int e) {
                const int i = e / kv, q = e - i * kv;
                return reinterpret_cast<const uint4 *>(Bi + (int64_t)(n0 + i) * ld)[q];
            },
            [&](int e, uint4 x) {
                const int i = e / kv, q = e - i * kv;
                reinterpret_cast<uint4 *>(P + (int64_t)i * kp)[q] = x;
            });
        __syncthreads();
        if (!backward) {
            for (int e = tid; e < nr * nrhs; e += nt) {
                const int i = e / nrhs, r = e - i * nrhs;
                T s = T(0);
                const T *row = P + (int64_t)i * kp;
#pragma unroll 4
                for (int k = 0; k <= n0 + i; k++) s += (cjp ? conj_v(row[k]) : row[k]) * v[k * nrhs + r];
                if (ldl) {
                    const T d = D[(int64_t)(n0 + i) * ld + n0 + i];
                    s = s * (cjp ? conj_v(d) : d);
                }
                Bg[(int64_t)r * ldb + fc + n0 + i] = s;
            }
        } else {
            for (int e = tid; e < kmax * nrhs; e += nt) {
                const int k = e / nrhs, r = e - k * nrhs;
                T s = T(0);
#pragma unroll 4
                for (int i = max(0, k - n0); i < nr; i++) s += P[(int64_t)i * kp + k] * v[(n0 + i) * nrhs + r];
                outp[e] += s;
            }
        }
    }
    if (backward) {
        __syncthreads();
        for (int e = tid; e < w * nrhs; e += nt) {
            const int j = e / nrhs, r = e - j * nrhs;
            Bg[(int64_t)r * ldb + fc + j] = outp[e];
        }
    }
}

// Forward product with the inverse for 1, 2, 4 or 8 right-hand sides: one warp
// per row n of Bi, lanes across k in 16-byte vectors read straight from
// global memory (no staging), the warp's partial sums reduced by shuffles:
// B[fc + n] = sum_{k <= n} op(Bi[n][k]) v[k] (times d_n for LDL).
template <typename T, int NR>
__device__ void diag_solve_inverse_fwd_warp(const T *__restrict__ Bi, const T *__restrict__ D, int w, int ld,
                                            bool ldl, bool cjp, const T *__restrict__ v, T *__restrict__ Bg,
                                            int64_t ldb, int fc) {
    constexpr int VEC = 16 / sizeof(T);
    // RU rows per warp at a time (n0, n0 + nw, ...): their loads are in flight
    // together, so a warp waits one memory latency per RU rows (RU bounded so
    // that the 1024-thread kernel stays within its 64 registers)
    constexpr int RU = sizeof(T) * NR <= 8 ? 4 : (sizeof(T) * NR <= 16 ? 2 : 1);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int n0 = warp; n0 < w; n0 += nw * RU) {
        const int nlast = min(w - 1, n0 + (RU - 1) * nw);
        T acc[RU][NR];
#pragma unroll
        for (int t = 0; t < RU; t++)
#pragma unroll
            for (int r = 0; r < NR; r++) acc[t][r] = T(0);
        for (int k0 = lane * VEC; k0 <= nlast; k0 += 32 * VEC) {
            uint4 u[RU];
#pragma unroll
            for (int t = 0; t < RU; t++) {
                const int n = n0 + t * nw;
                u[t] = (n < w && k0 <= n) ? __ldg(reinterpret_cast<const uint4 *>(Bi + (int64_t)n * ld + k0))
                                          : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int t = 0; t < RU; t++) {
                const int n = n0 + t * nw;
                T e[VEC];
                memcpy(e, &u[t], 16);
#pragma unroll
                for (int q = 0; q < VEC; q++) {
                    const int k = k0 + q;
                    if (k <= n) {
                        const T b = cjp ? conj_v(e[q]) : e[q];
#pragma unroll
                        for (int r = 0; r < NR; r++) acc[t][r] += b * v[k * NR + r];
                    }
                }
            }
        }
#pragma unroll
        for (int t = 0; t < RU; t++)
#pragma unroll
            for (int r = 0; r < NR; r++) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[t][r] += shfl_xor_v(acc[t][r], o);
            }
        if (lane == 0) {
#pragma unroll
            for (int t = 0; t < RU; t++) {
                const int n = n0 + t * nw;
                if (n < w) {
                    T d = T(1);
                    if (ldl) {
                        d = D[(int64_t)n * ld + n];
                        if (cjp) d = conj_v(d);
                    }
#pragma unroll
                    for (int r = 0; r < NR; r++) Bg[(int64_t)r * ldb + fc + n] = ldl ? acc[t][r] * d : acc[t][r];
                }
            }
        }
    }
}

// Backward product with the inverse for 1 or 2 right-hand sides:
// x[k] = sum_{n >= k} Bi[n][k] v'[n] (v' = d v for LDL).  One warp per row
// n, each lane accumulating its k-vectors (KS of them, w <= 32 KS VEC) in
// registers; the warps' partial sums meet in shared memory (atomics), then
// B[fc + k] = x[k].  xacc: [w][NR] shared accumulators.
template <typename T, int NR, int KS>
__device__ void diag_solve_inverse_bwd_warp(const T *__restrict__ Bi, const T *__restrict__ D, int w, int ld,
                                            bool ldl, const T *__restrict__ v, T *__restrict__ xacc,
                                            T *__restrict__ Bg, int64_t ldb, int fc) {
    constexpr int VEC = 16 / sizeof(T);
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int e = tid; e < w * NR; e += nt) xacc[e] = T(0);
    T part[KS][VEC][NR];
#pragma unroll
    for (int q = 0; q < KS; q++)
#pragma unroll
        for (int u = 0; u < VEC; u++)
#pragma unroll
            for (int r = 0; r < NR; r++) part[q][u][r] = T(0);
    __syncthreads();
    for (int n = warp; n < w; n += nw) {
        T vn[NR];
        const T dn = ldl ? D[(int64_t)n * ld + n] : T(1);
#pragma unroll
        for (int r = 0; r < NR; r++) vn[r] = ldl ? v[n * NR + r] * dn : v[n * NR + r];
        const T *row = Bi + (int64_t)n * ld;
#pragma unroll
        for (int q = 0; q < KS; q++) {
            const int k0 = (lane + 32 * q) * VEC;
            if (k0 <= n) {
                const uint4 u4 = __ldg(reinterpret_cast<const uint4 *>(row + k0));
                T e[VEC];
                memcpy(e, &u4, 16);
#pragma unroll
                for (int u = 0; u < VEC; u++)
                    if (k0 + u <= n)
#pragma unroll
                        for (int r = 0; r < NR; r++) part[q][u][r] += e[u] * vn[r];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < KS; q++)
#pragma unroll
        for (int u = 0; u < VEC; u++) {
            const int k = (lane + 32 * q) * VEC + u;
            if (k < w && k <= warp + (w - 1 - warp) / nw * nw)   // this warp saw a row n >= k
#pragma unroll
                for (int r = 0; r < NR; r++) atomic_add(&xacc[k * NR + r], part[q][u][r]);
        }
    __syncthreads();
    for (int e = tid; e < w * NR; e += nt) {
        const int k = e / NR, r = e - k * NR;
        Bg[(int64_t)r * ldb + fc + k] = xacc[e];
    }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_fwd_diag(Meta m, const int *__restrict__ cblks, const T *__restrict__ coefL,
                                                  T *__restrict__ B, int ldb, int nrhs, int unit, int pch,
                                                  const T *__restrict__ inv, int ldl, int cjp, int ipch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *y = reinterpret_cast<T *>(smem_raw);   // [w][nrhs]
    const int c = cblks[blockIdx.x];
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c];
    const T *D = coefL + m.coefoff[c];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    batched_copy(
        w * nrhs, tid, nt, [&](int e) { const int j = e / nrhs, r = e - j * nrhs; return B[(int64_t)r * ldb + fc + j]; },
        [&](int e, T v) { y[e] = v; });
    if (inv && m.invoff[c] >= 0) {
        // LU: the unit-lower inverse is the cblk's second one; the staged
        // rows start on a 16-byte boundary (vector stores)
        __syncthreads();
        const T *Bi = inv + m.invoff[c] + (unit && !ldl ? inv_span(w, ld) : 0);
        switch (nrhs) {
        case 1: diag_solve_inverse_fwd_warp<T, 1>(Bi, D, w, ld, ldl != 0, cjp != 0, y, B, ldb, fc); return;
        case 2: diag_solve_inverse_fwd_warp<T, 2>(Bi, D, w, ld, ldl != 0, cjp != 0, y, B, ldb, fc); return;
        case 4: diag_solve_inverse_fwd_warp<T, 4>(Bi, D, w, ld, ldl != 0, cjp != 0, y, B, ldb, fc); return;
        case 8: diag_solve_inverse_fwd_warp<T, 8>(Bi, D, w, ld, ldl != 0, cjp != 0, y, B, ldb, fc); return;
        default: break;
        }
        diag_solve_inverse<T>(Bi, D, w, ld, nrhs, false, ldl != 0, cjp != 0, y, nullptr,
                              y + align16_elems<T>((size_t)w * nrhs), ipch, B, ldb, fc);
        return;
    }
    T *tile = y + w * nrhs;                   // [32][33] diagonal tile
    T *P = tile + 32 * 33;                    // [pch][33] column panel below the tile
    for (int jb = 0; jb < w; jb += 32) {
        const int nb = min(32, w - jb);
        batched_copy(
            nb * nb, tid, nt, [&](int e) { const int i = e / nb, j = e - i * nb; return D[(int64_t)(jb + i) * ld + jb + j]; },
            [&](int e, T v) { const int i = e / nb, j = e - i * nb; tile[i * 33 + j] = v; });
        __syncthreads();
        if (tid < 32) {
            const T dinv = (lane < nb) ? T(1) / tile[lane * 33 + lane] : T(1);
            for (int r = 0; r < nrhs; r++) {
                T v = (lane < nb) ? y[(jb + lane) * nrhs + r] : T(0);
                for (int j = 0; j < nb; j++) {
                    if (!unit && lane == j) v *= dinv;
                    const T xj = shfl_v(v, j);
                    if (lane > j && lane < nb) v -= tile[lane * 33 + j] * xj;
                }
                if (lane < nb) y[(jb + lane) * nrhs + r] = v;
            }
        }
        __syncthreads();
        for (int r0 = jb + nb; r0 < w; r0 += pch) {
            const int nr = min(pch, w - r0);
            batched_copy(
                nr * nb, tid, nt, [&](int e) { const int i = e / nb, l = e - i * nb; return D[(int64_t)(r0 + i) * ld + jb + l]; },
                [&](int e, T v) { const int i = e / nb, l = e - i * nb; P[i * 33 + l] = v; });
            __syncthreads();
            for (int e = tid; e < nr * nrhs; e += nt) {
                const int i = e / nrhs, r = e - i * nrhs;
                T s = T(0);
#pragma unroll 8
                for (int l = 0; l < nb; l++) s += P[i * 33 + l] * y[(jb + l) * nrhs + r];
                y[(r0 + i) * nrhs + r] -= s;
            }
            __syncthreads();
        }
    }
    for (int e = tid; e < w * nrhs; e += nt) {
        int j = e / nrhs, r = e - j * nrhs;
        B[(int64_t)r * ldb + fc + j] = y[e];
    }
}

// ---------------------------------------------------------------------------
// Forward, off-diagonal part (kernels/solve_ztrsmsp.c:159 solve_blok_zgemm,
// Left, NoTrans): for every panel row i >= w of cblk c,
// B[row_i, :] -= P[i, :] . B[fcol:fcol+w, :].  One warp per panel row, lanes
// along the row (coalesced); cblks of one level can share target rows, so
// the subtraction is atomic.  chunks[i] = {cblk, first panel row}.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_fwd_off(Meta m, const int2 *__restrict__ chunks, const T *__restrict__ coef,
                                                 T *__restrict__ B, int ldb, int nrhs, int rows_per_chunk) {
    // the chunk's rows are staged in shared memory with 16-byte vector
    // loads (one burst), then one warp per row reads them from there
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int VEC = 16 / sizeof(T);
    const int2 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const int wv = (w + VEC - 1) / VEC, wp = wv * VEC;
    const int rend = min(h, r0 + rows_per_chunk), nr = rend - r0;
    T *y = reinterpret_cast<T *>(smem_raw);            // [nrhs][wp] (zero padded)
    T *Pr = y + align16_elems<T>((size_t)nrhs * wp);    // [nr][wp]
    const int tid = threadIdx.x, nt = blockDim.x;
    const T *P = coef + m.coefoff[c] + (int64_t)r0 * ld;
    batched_copy<4>(
        nr * wv, tid, nt, [&](int e) { const int i = e / wv, q = e - i * wv; return reinterpret_cast<const uint4 *>(P + (int64_t)i * ld)[q]; },
        [&](int e, uint4 v) { const int i = e / wv, q = e - i * wv; reinterpret_cast<uint4 *>(Pr + (int64_t)i * wp)[q] = v; });
    batched_copy(
        nrhs * wp, tid, nt,
        [&](int e) { const int r = e / wp, j = e - r * wp; return j < w ? B[(int64_t)r * ldb + fc + j] : T(0); },
        [&](int e, T v) { y[e] = v; });
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int i = warp; i < nr; i += nw) {
        const T *row = Pr + (int64_t)i * wp;
        const int grow = m.rowidx[m.rowbase[c] + r0 + i];
        for (int r = 0; r < nrhs; r++) {
            T s = T(0);
            for (int j = lane; j < w; j += 32) s += row[j] * y[r * wp + j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += shfl_xor_v(s, o);
            if (lane == 0) atomic_sub(&B[(int64_t)r * ldb + grow], s);
        }
    }
}

// ---------------------------------------------------------------------------
// Backward, off-diagonal gather (kernels/solve_ztrsmsp.c:450
// solve_cblk_ztrsmsp_backward walks browtab): B[fcol+j, :] -= sum_i op(P[i, j])
// B[row_i, :] over panel rows i >= w of cblk c (P = L for POTRF / LDL, U^T
// for GETRF; op = conj for the Hermitian forms when cjp).  The chunk's rows
// are staged in shared memory (16-byte vector loads), then one thread per
// column sums them; partial sums of the chunks are combined atomically.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_bwd_off(Meta m, const int2 *__restrict__ chunks, const T *__restrict__ coef,
                                                 T *__restrict__ B, int ldb, int nrhs, int rows_per_chunk, int cjp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int VEC = 16 / sizeof(T);
    const int2 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const int wv = (w + VEC - 1) / VEC, wp = wv * VEC;
    const int rend = min(h, r0 + rows_per_chunk), nr = rend - r0;
    T *xr = reinterpret_cast<T *>(smem_raw);            // [rows][nrhs]: the solution at the chunk's rows
    T *Pr = xr + align16_elems<T>((size_t)rows_per_chunk * nrhs);   // [nr][wp]
    const int tid = threadIdx.x, nt = blockDim.x;
    const T *P = coef + m.coefoff[c] + (int64_t)r0 * ld;
    batched_copy<4>(
        nr * wv, tid, nt, [&](int e) { const int i = e / wv, q = e - i * wv; return reinterpret_cast<const uint4 *>(P + (int64_t)i * ld)[q]; },
        [&](int e, uint4 v) { const int i = e / wv, q = e - i * wv; reinterpret_cast<uint4 *>(Pr + (int64_t)i * wp)[q] = v; });
    batched_copy(
        nr * nrhs, tid, nt,
        [&](int e) { const int i = e / nrhs, r = e - i * nrhs; return B[(int64_t)r * ldb + m.rowidx[m.rowbase[c] + r0 + i]]; },
        [&](int e, T v) { xr[e] = v; });
    __syncthreads();
    for (int e = tid; e < w * nrhs; e += nt) {
        const int j = e % w, r = e / w;
        T s = T(0);
#pragma unroll 8
        for (int i = 0; i < nr; i++) {
            const T v = Pr[(int64_t)i * wp + j];
            s += (cjp ? conj_v(v) : v) * xr[i * nrhs + r];
        }
        atomic_sub(&B[(int64_t)r * ldb + fc + j], s);
    }
}

// ---------------------------------------------------------------------------
// Off-diagonal kernels for 1, 2, 4 or 8 right-hand sides, the panel rows read
// straight from global memory in 16-byte vectors (no shared staging), so a
// chunk costs about one memory latency:
//   k_fwd_off_direct: one warp per RU rows at a time (all RU rows' loads in
//     flight together), lanes across the columns, the cblk's solution in
//     shared memory (zero padded); the row sums are reduced by shuffles and
//     subtracted atomically from B at the rows' global indices;
//   k_bwd_off_direct (2 or 4 right-hand sides): one thread per column,
//     looping over the chunk's rows (coalesced across the threads), the
//     solution at those rows gathered in shared memory; partial sums of the
//     chunks meet atomically.  (One right-hand side keeps k_bwd_off: its
//     16-byte staging wins when each loaded value feeds a single product.)
// Same products as k_fwd_off / k_bwd_off.
// ---------------------------------------------------------------------------
template <typename T, int NR>
__global__ void __launch_bounds__(256) k_fwd_off_direct(Meta m, const int2 *__restrict__ chunks,
                                                        const T *__restrict__ coef, T *__restrict__ B, int ldb,
                                                        int rows_per_chunk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int VEC = 16 / sizeof(T), RU = 4;
    const int2 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const int wp = (w + VEC - 1) / VEC * VEC;
    const int nr = min(h, r0 + rows_per_chunk) - r0;
    T *y = reinterpret_cast<T *>(smem_raw);            // [wp][NR] (zero padded)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int e = tid; e < wp * NR; e += blockDim.x) {
        const int j = e / NR, r = e - j * NR;
        y[e] = j < w ? B[(int64_t)r * ldb + fc + j] : T(0);
    }
    __syncthreads();
    const T *P = coef + m.coefoff[c] + (int64_t)r0 * ld;
    const int *rows = m.rowidx + m.rowbase[c] + r0;
    for (int i0 = warp * RU; i0 < nr; i0 += nw * RU) {
        T acc[RU][NR];
#pragma unroll
        for (int u = 0; u < RU; u++)
#pragma unroll
            for (int r = 0; r < NR; r++) acc[u][r] = T(0);
        for (int k0 = lane * VEC; k0 < wp; k0 += 32 * VEC) {
            T e[RU][VEC];
#pragma unroll
            for (int u = 0; u < RU; u++) {
                // rows past the chunk read row i0 again (discarded below)
                const int i = (i0 + u < nr) ? i0 + u : i0;
                const uint4 v4 = __ldg(reinterpret_cast<const uint4 *>(P + (int64_t)i * ld + k0));
                memcpy(e[u], &v4, 16);
            }
#pragma unroll
            for (int q = 0; q < VEC; q++) {
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const T yk = y[(k0 + q) * NR + r];
#pragma unroll
                    for (int u = 0; u < RU; u++) acc[u][r] += e[u][q] * yk;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < RU; u++)
#pragma unroll
            for (int r = 0; r < NR; r++) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[u][r] += shfl_xor_v(acc[u][r], o);
            }
        if (lane == 0)
#pragma unroll
            for (int u = 0; u < RU; u++)
                if (i0 + u < nr)
#pragma unroll
                    for (int r = 0; r < NR; r++) atomic_sub(&B[(int64_t)r * ldb + rows[i0 + u]], acc[u][r]);
    }
}

template <typename T, int NR>
__global__ void __launch_bounds__(256) k_bwd_off_direct(Meta m, const int2 *__restrict__ chunks,
                                                        const T *__restrict__ coef, T *__restrict__ B, int ldb,
                                                        int rows_per_chunk, int cjp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int2 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const int nr = min(h, r0 + rows_per_chunk) - r0;
    T *xr = reinterpret_cast<T *>(smem_raw);            // [rows][NR]: the solution at the chunk's rows
    const int tid = threadIdx.x, nt = blockDim.x;
    const int *rows = m.rowidx + m.rowbase[c] + r0;
    for (int e = tid; e < nr * NR; e += nt) {
        const int i = e / NR, r = e - i * NR;
        xr[e] = B[(int64_t)r * ldb + rows[i]];
    }
    __syncthreads();
    const T *P = coef + m.coefoff[c] + (int64_t)r0 * ld;
    for (int j = tid; j < w; j += nt) {
        T acc[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) acc[r] = T(0);
#pragma unroll 8
        for (int i = 0; i < nr; i++) {
            T pv = P[(int64_t)i * ld + j];
            if (cjp) pv = conj_v(pv);
#pragma unroll
            for (int r = 0; r < NR; r++) acc[r] += pv * xr[i * NR + r];
        }
#pragma unroll
        for (int r = 0; r < NR; r++) atomic_sub(&B[(int64_t)r * ldb + fc + j], acc[r]);
    }
}

// ---------------------------------------------------------------------------
// Levels of narrow cblks (w <= 32, no diagonal-block inverse: the leaves of
// the elimination tree, tens of thousands of them): one warp per cblk does
// the diagonal solve and its off-diagonal rows in one launch, the solution
// of the cblk kept in the lanes' registers (lane j holds x_j) and handed
// to the row products by shuffles.  Same operations as k_fwd_diag +
// k_fwd_off (forward) and k_bwd_off + k_bwd_diag (backward) for these
// cblks; the backward gather needs no atomics (one warp owns the cblk).
// ---------------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 1) k_fwd_small(Meta m, const int *__restrict__ cblks, int ncb,
                                                   const T *__restrict__ coefL, T *__restrict__ B, int ldb, int nrhs,
                                                   int unit) {
    // R right-hand sides at a time (nrhs a multiple of R), each one's
    // operations in the same order as alone
    constexpr int VK = 16 / sizeof(T);
    __shared__ __align__(16) unsigned char xs_raw[8 * 32 * R * sizeof(T)];
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= ncb) return;                                  // whole warps
    T *xs = reinterpret_cast<T *>(xs_raw) + (threadIdx.x >> 5) * 32 * R;   // [32][R]: x of this cblk
    const int c = cblks[q];
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const T *D = coefL + m.coefoff[c];
    const T dinv = (lane < w && !unit) ? T(1) / D[(int64_t)lane * ld + lane] : T(1);
    const int *rows = m.rowidx + m.rowbase[c];
    for (int r0 = 0; r0 < nrhs; r0 += R) {
        T v[R];
#pragma unroll
        for (int u = 0; u < R; u++) v[u] = (lane < w) ? B[(int64_t)(r0 + u) * ldb + fc + lane] : T(0);
        for (int j = 0; j < w; j++) {
            const T lj = (lane > j && lane < w) ? D[(int64_t)lane * ld + j] : T(0);
#pragma unroll
            for (int u = 0; u < R; u++) {
                if (lane == j) v[u] = v[u] * dinv;
                const T xj = shfl_v(v[u], j);
                if (lane > j && lane < w) v[u] -= lj * xj;
            }
        }
        if (lane < w)
#pragma unroll
            for (int u = 0; u < R; u++) B[(int64_t)(r0 + u) * ldb + fc + lane] = v[u];
        __syncwarp();
#pragma unroll
        for (int u = 0; u < R; u++) xs[lane * R + u] = v[u];   // zero past w
        __syncwarp();
        // off-diagonal rows, lane = row: 16-byte loads of the row (rows are
        // 16-byte aligned, ld >= w rounded to 4), x_j broadcast from shared
        for (int i0 = w; i0 < h; i0 += 32) {
            const int i = i0 + lane;
            const T *row = D + (int64_t)(i < h ? i : i0) * ld;
            T sacc[R];
#pragma unroll
            for (int u = 0; u < R; u++) sacc[u] = T(0);
            for (int j0 = 0; j0 < w; j0 += VK) {
                T e[VK];
                const uint4 v4 = *reinterpret_cast<const uint4 *>(row + j0);
                memcpy(e, &v4, 16);
#pragma unroll
                for (int t = 0; t < VK; t++)
                    if (j0 + t < w)
#pragma unroll
                        for (int u = 0; u < R; u++) sacc[u] += e[t] * xs[(j0 + t) * R + u];
            }
            if (i < h)
#pragma unroll
                for (int u = 0; u < R; u++) atomic_sub(&B[(int64_t)(r0 + u) * ldb + rows[i]], sacc[u]);
        }
        __syncwarp();
    }
}

// upper != 0: U of the LU diagonal block (row-major upper part, non-unit),
// P = the U^t panel (coefP); else op(L)^t with op = conj when cjp, P = L.
template <typename T, int R>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 1) k_bwd_small(Meta m, const int *__restrict__ cblks, int ncb,
                                                   const T *__restrict__ coefL, const T *__restrict__ coefP,
                                                   T *__restrict__ B, int ldb, int nrhs, int upper, int unit,
                                                   int cjp) {
    __shared__ __align__(16) unsigned char xs_raw[8 * 32 * R * sizeof(T)];
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= ncb) return;
    T *xs = reinterpret_cast<T *>(xs_raw) + (threadIdx.x >> 5) * 32 * R;   // [32][R]: x at 32 panel rows
    const int c = cblks[q];
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const T *D = coefL + m.coefoff[c];
    const T *P = coefP + m.coefoff[c];
    const int *rows = m.rowidx + m.rowbase[c];
    T dinv = T(1);
    if (lane < w && !unit) {
        const T d = D[(int64_t)lane * ld + lane];
        dinv = T(1) / (cjp ? conj_v(d) : d);
    }
    for (int r0 = 0; r0 < nrhs; r0 += R) {
        // gather: x_j -= sum_i op(P[i][j]) x[row_i]; the x of 32 rows at a
        // time are fetched by the lanes (independent loads) into shared
        // memory, then summed in increasing i as one lane per column
        T sacc[R];
#pragma unroll
        for (int u = 0; u < R; u++) sacc[u] = T(0);
        for (int i0 = w; i0 < h; i0 += 32) {
            const int nr = min(32, h - i0);
            if (lane < nr) {
                const int gi = rows[i0 + lane];
#pragma unroll
                for (int u = 0; u < R; u++) xs[lane * R + u] = B[(int64_t)(r0 + u) * ldb + gi];
            }
            __syncwarp();
            if (lane < w) {
                const T *pr = P + (int64_t)i0 * ld + lane;
#pragma unroll 4
                for (int t = 0; t < nr; t++) {
                    T pv = pr[(int64_t)t * ld];
                    if (cjp) pv = conj_v(pv);
#pragma unroll
                    for (int u = 0; u < R; u++) sacc[u] += pv * xs[t * R + u];
                }
            }
            __syncwarp();
        }
        T v[R];
#pragma unroll
        for (int u = 0; u < R; u++) v[u] = (lane < w) ? B[(int64_t)(r0 + u) * ldb + fc + lane] - sacc[u] : T(0);
        for (int j = w - 1; j >= 0; j--) {
            T dlj = T(0);
            if (lane < j) {
                if (upper) dlj = D[(int64_t)lane * ld + j];
                else {
                    dlj = D[(int64_t)j * ld + lane];
                    if (cjp) dlj = conj_v(dlj);
                }
            }
#pragma unroll
            for (int u = 0; u < R; u++) {
                if (lane == j) v[u] = v[u] * dinv;
                const T xj = shfl_v(v[u], j);
                if (lane < j) v[u] -= dlj * xj;
            }
        }
        if (lane < w)
#pragma unroll
            for (int u = 0; u < R; u++) B[(int64_t)(r0 + u) * ldb + fc + lane] = v[u];
    }
}

// ---------------------------------------------------------------------------
// Backward, diagonal part: B[fcol:fcol+w, :] := D^{-1} B[...] with
// D = op(L_kk)^t (POTRF: Left, Lower, ConjTrans, NonUnit; LDL: the unit
// lower part, Left, Lower, ConjTrans/Trans, Unit, after k_diag_scale) or the
// upper triangle U_kk of the LU diagonal block (Left, Upper, NoTrans,
// NonUnit).  op = conj when cjp.  Blocked by 32 columns from the last block
// up: warp 0 substitutes through the tile, then all threads update the rows
// above from the tile's panel staged in shared memory (pch rows at a time).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(1024) k_bwd_diag(Meta m, const int *__restrict__ cblks, const T *__restrict__ coefL,
                                                  T *__restrict__ B, int ldb, int nrhs, int upper, int unit, int cjp,
                                                  int pch, const T *__restrict__ inv, int ldl, int ipch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *x = reinterpret_cast<T *>(smem_raw);   // [w][nrhs]
    const int c = cblks[blockIdx.x];
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c];
    const T *D = coefL + m.coefoff[c];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    batched_copy(
        w * nrhs, tid, nt, [&](int e) { const int j = e / nrhs, r = e - j * nrhs; return B[(int64_t)r * ldb + fc + j]; },
        [&](int e, T v) { x[e] = v; });
    if (inv && m.invoff[c] >= 0) {
        __syncthreads();
        const T *Bi = inv + m.invoff[c];
        constexpr int VEC = 16 / sizeof(T);
        T *acc = x + (size_t)w * nrhs;
        // register budget of the 1024-thread block: KS VEC NR elements of T per lane
        if (nrhs == 1 && w <= 32 * 4 * VEC) {
            diag_solve_inverse_bwd_warp<T, 1, 4>(Bi, D, w, ld, ldl != 0, x, acc, B, ldb, fc);
            return;
        }
        if (nrhs == 1 && w <= 32 * 8 * VEC && sizeof(T) * 8 * VEC <= 128) {
            diag_solve_inverse_bwd_warp<T, 1, 8>(Bi, D, w, ld, ldl != 0, x, acc, B, ldb, fc);
            return;
        }
        if (nrhs == 2 && w <= 32 * 4 * VEC && sizeof(T) * 8 * VEC <= 128) {
            diag_solve_inverse_bwd_warp<T, 2, 4>(Bi, D, w, ld, ldl != 0, x, acc, B, ldb, fc);
            return;
        }
        diag_solve_inverse<T>(Bi, D, w, ld, nrhs, true, ldl != 0, false, x, acc,
                              x + align16_elems<T>((size_t)2 * w * nrhs), ipch, B, ldb, fc);
        return;
    }
    T *tile = x + w * nrhs;                   // [32][33] diagonal tile (op applied)
    T *P = tile + 32 * 33;                    // [pch][33]: coefficients of the rows above
    const int nblk = (w + 31) / 32;
    for (int bi = nblk - 1; bi >= 0; bi--) {
        const int jb = bi * 32, nb = min(32, w - jb);
        batched_copy(
            nb * nb, tid, nt,
            [&](int e) {
                const int i = e / nb, j = e - i * nb;
                const T v = D[(int64_t)(jb + i) * ld + jb + j];
                return cjp ? conj_v(v) : v;
            },
            [&](int e, T v) { const int i = e / nb, j = e - i * nb; tile[i * 33 + j] = v; });
        __syncthreads();
        if (tid < 32) {
            const T dinv = (lane < nb && !unit) ? T(1) / tile[lane * 33 + lane] : T(1);
            for (int r = 0; r < nrhs; r++) {
                T v = (lane < nb) ? x[(jb + lane) * nrhs + r] : T(0);
                for (int j = nb - 1; j >= 0; j--) {
                    if (lane == j) v = v * dinv;
                    const T xj = shfl_v(v, j);
                    if (lane < j) {
                        // upper: U[l][j]; Cholesky / LDL: op(L)^t[l][j] = op(L[j][l])
                        const T dlj = upper ? tile[lane * 33 + j] : tile[j * 33 + lane];
                        v -= dlj * xj;
                    }
                }
                if (lane < nb) x[(jb + lane) * nrhs + r] = v;
            }
        }
        __syncthreads();
        for (int r0 = 0; r0 < jb; r0 += pch) {
            const int nr = min(pch, jb - r0);
            // P[i][l] = coefficient of x[jb + l] in row r0 + i
            if (upper) {
                batched_copy(
                    nr * nb, tid, nt, [&](int e) { const int i = e / nb, l = e - i * nb; return D[(int64_t)(r0 + i) * ld + jb + l]; },
                    [&](int e, T v) { const int i = e / nb, l = e - i * nb; P[i * 33 + l] = v; });
            } else {
                batched_copy(
                    nr * nb, tid, nt,
                    [&](int e) {
                        const int l = e / nr, i = e - l * nr;
                        const T v = D[(int64_t)(jb + l) * ld + r0 + i];
                        return cjp ? conj_v(v) : v;
                    },
                    [&](int e, T v) { const int l = e / nr, i = e - l * nr; P[i * 33 + l] = v; });
            }
            __syncthreads();
            for (int e = tid; e < nr * nrhs; e += nt) {
                const int i = e / nrhs, r = e - i * nrhs;
                T s = T(0);
#pragma unroll 8
                for (int l = 0; l < nb; l++) s += P[i * 33 + l] * x[(jb + l) * nrhs + r];
                x[(r0 + i) * nrhs + r] -= s;
            }
            __syncthreads();
        }
    }
    for (int e = tid; e < w * nrhs; e += nt) {
        int j = e / nrhs, r = e - j * nrhs;
        B[(int64_t)r * ldb + fc + j] = x[e];
    }
}

// ---------------------------------------------------------------------------
// Diagonal solve of the LDL forms (kernels/solve_ztrsmsp.c:630
// solve_cblk_zdiag): B[fcol + j, :] /= D_jj, one CTA per cblk (grid-strided).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_diag_scale(Meta m, const T *__restrict__ coefL, T *__restrict__ B, int ldb, int nrhs) {
    for (int c = blockIdx.x; c < m.cblknbr; c += gridDim.x) {
        const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c];
        const T *D = coefL + m.coefoff[c];
        for (int e = threadIdx.x; e < w * nrhs; e += blockDim.x) {
            const int j = e % w, r = e / w;
            T &v = B[(int64_t)r * ldb + fc + j];
            v = v * (T(1) / D[(int64_t)j * ld + j]);
        }
    }
}

// ---------------------------------------------------------------------------
// Right-hand-side permutation (bcsc/bvec_zlapmr.c:816 bvec_zlapmr):
// forward  Y[k] = X[peritab[k]] (user order -> factor order), backward
// X[peritab[k]] = Y[k].  Converts the precision on the way.
// ---------------------------------------------------------------------------
template <typename Tin, typename Tout>
__global__ void k_permute(int n, int nrhs, const int *__restrict__ peritab, const Tin *__restrict__ X,
                          int64_t ldx, Tout *__restrict__ Y, int64_t ldy, int backward) {
    // one thread per row index: the permutation entry is read once for all
    // right-hand sides, whose copies are independent loads in flight
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int p = peritab ? peritab[k] : k;   // no table: the identity (a cast copy)
        const int64_t src = backward ? k : p, dst = backward ? p : k;
#pragma unroll 4
        for (int r = 0; r < nrhs; r++) Y[r * ldy + dst] = (Tout)X[r * ldx + src];
    }
}

template <typename Tin, typename Tout>
__global__ void k_convert(int64_t n, const Tin *__restrict__ x, Tout *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] = (Tout)x[i];
}

// ---------------------------------------------------------------------------
// Refinement vector kernels, FP64 real (S = double) or complex (S = cdouble)
// (bcsc/bcsc_zspmv.c:629 bcsc_zspmv on the permuted matrix held as CSR, one
// warp per row; bvec_z{dotc,nrm2,axpy,scal,copy,gemv}, bcsc/bvec_zcompute.c).
// Reductions go through per-CTA partials finished by one CTA, so results are
// deterministic.
// ---------------------------------------------------------------------------
template <typename S>
__global__ void k_spmv(int n, const int64_t *__restrict__ rowptr, const int *__restrict__ col,
                       const S *__restrict__ val, double alpha, const S *__restrict__ x,
                       double beta, S *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (; row < n; row += nwarps) {
        S s = S(0.0);
        for (int64_t k = rowptr[row] + lane; k < rowptr[row + 1]; k += 32) s += val[k] * x[col[k]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += shfl_xor_v(s, o);
        if (lane == 0) y[row] = alpha * s + (beta == 0.0 ? S(0.0) : beta * y[row]);
    }
}

constexpr int RED_THREADS = 256;

template <typename S>
__device__ __forceinline__ S block_sum(S v, S *sh) {
    for (int o = 16; o > 0; o >>= 1) v += shfl_xor_v(v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : S(0.0);
    if (warp == 0)
        for (int o = 16; o > 0; o >>= 1) v += shfl_xor_v(v, o);
    return v;
}

// partial[blockIdx] = sum conj(x) y (bvec_zdotc), or sum |x|^2 when y == nullptr
template <typename S>
__global__ void k_dot_partial(int64_t n, const S *__restrict__ x, const S *__restrict__ y, S *__restrict__ partial) {
    __shared__ S sh[32];
    S s = S(0.0);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += y ? conj_v(x[i]) * y[i] : S(abs2_v(x[i]));
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// *out = sum of the partials (do_sqrt: sqrt of its real part, for norms)
template <typename S>
__global__ void k_dot_final(int np, const S *__restrict__ partial, S *__restrict__ out, int do_sqrt) {
    __shared__ S sh[32];
    S s = S(0.0);
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) *out = do_sqrt ? S(sqrt(real_v(s))) : s;
}

template <typename S>
__global__ void k_axpy(int64_t n, S alpha, const S *__restrict__ x, S *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}

// p = z + beta * p
template <typename S>
__global__ void k_xpby(int64_t n, const S *__restrict__ z, S beta, S *__restrict__ p) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// y += sign * (*alpha) * x with the scalar read from device memory (GMRES
// orthogonalization without a host round trip per projection).
template <typename S>
__global__ void k_axpy_dev(int64_t n, const S *__restrict__ alpha, double sign, const S *__restrict__ x,
                           S *__restrict__ y) {
    const S a = sign * (*alpha);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

template <typename S>
__global__ void k_scal(int64_t n, double a, S *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] = a * x[i];
}

// x += W(:, 0:k) y  (bvec_zgemv, bcsc/bvec_zcompute.c; W column-major, ld ldw)
template <typename S>
__global__ void k_gemv_acc(int64_t n, int k, const S *__restrict__ W, int64_t ldw, const S *__restrict__ y,
                           S *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        S s = S(0.0);
        for (int j = 0; j < k; j++) s += W[i + j * ldw] * y[j];
        x[i] += s;
    }
}

// ---------------------------------------------------------------------------
// Multi-right-hand-side forms for the refinement run in lockstep on k <= 16
// columns (column-major, ld = n): each column keeps its own scalars, and
// each column's reductions follow exactly the single-column kernels' order,
// so a column's iterates are those of running it alone (the reference
// refines one right-hand side after the other, refinement/pastix_task_refine.c).
// ---------------------------------------------------------------------------
constexpr int MULTI_MAX = 16;
template <typename S> struct Coefs { S v[MULTI_MAX]; };

// partial[c * gridDim.x + b] = sum over the block's share of conj(x_c) y_c
// (|x_c|^2 when y == nullptr); blockIdx.y = column
template <typename S>
__global__ void k_dot_partial_multi(int64_t n, const S *__restrict__ x, const S *__restrict__ y,
                                    S *__restrict__ partial) {
    __shared__ S sh[32];
    const int c = blockIdx.y;
    const S *xc = x + (int64_t)c * n;
    const S *yc = y ? y + (int64_t)c * n : nullptr;
    S s = S(0.0);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += yc ? conj_v(xc[i]) * yc[i] : S(abs2_v(xc[i]));
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[(int64_t)c * gridDim.x + blockIdx.x] = s;
}

// out[c] = sum of column c's np partials (sqrt of the real part when do_sqrt)
template <typename S>
__global__ void k_dot_final_multi(int np, const S *__restrict__ partial, S *__restrict__ out, int do_sqrt) {
    __shared__ S sh[32];
    const int c = blockIdx.x;
    S s = S(0.0);
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[(int64_t)c * np + i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[c] = do_sqrt ? S(sqrt(real_v(s))) : s;
}

// y_c += a_c x_c (a from the parameter block)
template <typename S>
__global__ void k_axpy_multi(int64_t n, int k, Coefs<S> a, const S *__restrict__ x, S *__restrict__ y) {
    const int64_t tot = n * k;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
        y[e] += a.v[e / n] * x[e];
}

// y_c += sign * alpha[c] x_c with alpha in device memory (GMRES projections)
template <typename S>
__global__ void k_axpy_multi_dev(int64_t n, int k, const S *__restrict__ alpha, double sign, const S *__restrict__ x,
                                 S *__restrict__ y) {
    const int64_t tot = n * k;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
        y[e] += (sign * alpha[e / n]) * x[e];
}

// p_c = z_c + beta_c p_c
template <typename S>
__global__ void k_xpby_multi(int64_t n, int k, const S *__restrict__ z, Coefs<S> beta, S *__restrict__ p) {
    const int64_t tot = n * k;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
        p[e] = z[e] + beta.v[e / n] * p[e];
}

// x_c *= a_c
template <typename S>
__global__ void k_scal_multi(int64_t n, int k, Coefs<double> a, S *__restrict__ x) {
    const int64_t tot = n * k;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
        x[e] = a.v[e / n] * x[e];
}

// y_c = alpha A x_c + beta y_c on the permuted CSR, one warp per row, all
// columns from one pass over the row (same summation order per column as
// k_spmv)
// The same products with one thread per row (short rows, as the stencil
// matrices have: a warp per row would leave most lanes idle); the row's
// entries are summed in order.
template <typename S>
__global__ void k_spmv_rows_multi(int n, int k, const int64_t *__restrict__ rowptr, const int *__restrict__ col,
                                  const S *__restrict__ val, double alpha, const S *__restrict__ x, double beta,
                                  S *__restrict__ y) {
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        S s[MULTI_MAX];
#pragma unroll
        for (int c = 0; c < MULTI_MAX; c++) s[c] = S(0.0);
        const int64_t q1 = rowptr[row + 1];
        for (int64_t q = rowptr[row]; q < q1; q++) {
            const S v = val[q];
            const int cc = col[q];
#pragma unroll
            for (int c = 0; c < MULTI_MAX; c++)
                if (c < k) s[c] += v * x[(int64_t)c * n + cc];
        }
#pragma unroll
        for (int c = 0; c < MULTI_MAX; c++) {
            if (c >= k) break;
            S &yy = y[(int64_t)c * n + row];
            yy = alpha * s[c] + (beta == 0.0 ? S(0.0) : beta * yy);
        }
    }
}

template <typename S>
__global__ void k_spmv_multi(int n, int k, const int64_t *__restrict__ rowptr, const int *__restrict__ col,
                             const S *__restrict__ val, double alpha, const S *__restrict__ x, double beta,
                             S *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (; row < n; row += nwarps) {
        S s[MULTI_MAX];
#pragma unroll
        for (int c = 0; c < MULTI_MAX; c++) s[c] = S(0.0);
        for (int64_t q = rowptr[row] + lane; q < rowptr[row + 1]; q += 32) {
            const S v = val[q];
            const int cc = col[q];
#pragma unroll
            for (int c = 0; c < MULTI_MAX; c++)
                if (c < k) s[c] += v * x[(int64_t)c * n + cc];
        }
#pragma unroll
        for (int c = 0; c < MULTI_MAX; c++) {
            if (c >= k) break;
            S t = s[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += shfl_xor_v(t, o);
            if (lane == 0) {
                S &yy = y[(int64_t)c * n + row];
                yy = alpha * t + (beta == 0.0 ? S(0.0) : beta * yy);
            }
        }
    }
}

// out[c * nseg + s] = sum |x_c|^2 over segment s (blockIdx.y = column)
template <typename S>
__global__ void k_seg_sumsq_multi(int nseg, const int64_t *__restrict__ seg, int64_t n, const S *__restrict__ x,
                                  double *__restrict__ out) {
    __shared__ double sh[32];
    const int c = blockIdx.y;
    const S *xc = x + (int64_t)c * n;
    for (int sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        double v = 0.0;
        for (int64_t i = seg[sg] + threadIdx.x; i < seg[sg + 1]; i += blockDim.x) v += abs2_v(xc[i]);
        v = block_sum(v, sh);
        if (threadIdx.x == 0) out[(int64_t)c * nseg + sg] = v;
        __syncthreads();
    }
}

// Gather the permuted-matrix values from the user's values; src < 0 marks
// the mirrored entry of a Hermitian matrix (conj(vals[~src])).
template <typename S>
__global__ void k_gather_vals(int64_t nnz, const int64_t *__restrict__ src, const S *__restrict__ vals,
                              S *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = src[i];
        out[i] = (k < 0) ? conj_v(vals[~k]) : vals[k];
    }
}

// Static pivoting threshold from the matrix norm (sopalin/pastix_task_sopalin.c:
// 461-485): s[1] = -magn if magn < 0, eps * s[0] if magn == 0, magn * s[0]
// otherwise, with s[0] = ||A||_F.
__global__ void k_static_pivot_threshold(double *s, double magn, double eps) {
    const double anorm = s[0];
    s[1] = (magn < 0.) ? -magn : ((magn == 0.) ? eps * anorm : magn * anorm);
}

// Per-segment sum of squares: out[s] = sum |x_i|^2 over [seg[s], seg[s+1]).
template <typename S>
__global__ void k_seg_sumsq(int nseg, const int64_t *__restrict__ seg, const S *__restrict__ x,
                            double *__restrict__ out) {
    __shared__ double sh[32];
    for (int sg = blockIdx.x; sg < nseg; sg += gridDim.x) {
        double v = 0.0;
        for (int64_t i = seg[sg] + threadIdx.x; i < seg[sg + 1]; i += blockDim.x) v += abs2_v(x[i]);
        v = block_sum(v, sh);
        if (threadIdx.x == 0) out[sg] = v;
        __syncthreads();
    }
}

// Weighted sum of squares for the Frobenius norm (off-diagonal entries of a
// one-triangle symmetric matrix count twice).
template <typename S>
__global__ void k_sumsq_partial(int64_t nnz, const S *__restrict__ v, const int8_t *__restrict__ wgt,
                                double *__restrict__ partial) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (int64_t)gridDim.x * blockDim.x)
        s += (double)wgt[i] * abs2_v(v[i]);
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

}  // namespace pgpu
