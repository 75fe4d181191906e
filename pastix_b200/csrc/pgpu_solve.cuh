// Forward/backward supernodal triangular solves (kernels/solve_ztrsmsp.c) and
// the vector kernels of the iterative refinement (bcsc/bcsc_zspmv.c,
// bcsc/bvec_zcompute.c).  Right-hand sides are column-major n x nrhs in the
// permuted numbering.
#pragma once

#include "pgpu_common.cuh"

namespace pgpu {

constexpr int SOLVE_MAXRHS = 16;

// ---------------------------------------------------------------------------
// Forward, diagonal part (kernels/solve_ztrsmsp.c:75 solve_blok_ztrsm with
// Left, Lower, NoTrans): B[fcol:fcol+w, :] := D^{-1} B[...], D = L_kk
// (POTRF, non-unit) or the unit lower part of the LU diagonal block.  One CTA
// per cblk of the level, blocked by 32 columns: warp 0 substitutes through
// the 32x32 tile (shuffles, no block barrier), then all threads update the
// rows below inside the diagonal block.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_fwd_diag(Meta m, const int *__restrict__ cblks, const T *__restrict__ coefL,
                           T *__restrict__ B, int ldb, int nrhs, int unit) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *y = reinterpret_cast<T *>(smem_raw);   // [w][nrhs]
    const int c = cblks[blockIdx.x];
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c];
    const T *D = coefL + m.coefoff[c];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    for (int e = tid; e < w * nrhs; e += nt) {
        int j = e / nrhs, r = e - j * nrhs;
        y[e] = B[(int64_t)r * ldb + fc + j];
    }
    __syncthreads();
    T *tile = y + w * nrhs;                   // [32][33] diagonal tile
    for (int jb = 0; jb < w; jb += 32) {
        const int nb = min(32, w - jb);
        for (int e = tid; e < nb * nb; e += nt) {
            const int i = e / nb, j = e - i * nb;
            tile[i * 33 + j] = D[(int64_t)(jb + i) * ld + jb + j];
        }
        __syncthreads();
        if (tid < 32) {
            const T dinv = (lane < nb) ? T(1) / tile[lane * 33 + lane] : T(1);
            for (int r = 0; r < nrhs; r++) {
                T v = (lane < nb) ? y[(jb + lane) * nrhs + r] : T(0);
                for (int j = 0; j < nb; j++) {
                    if (!unit && lane == j) v *= dinv;
                    const T xj = __shfl_sync(0xffffffffu, v, j);
                    if (lane > j && lane < nb) v -= tile[lane * 33 + j] * xj;
                }
                if (lane < nb) y[(jb + lane) * nrhs + r] = v;
            }
        }
        __syncthreads();
        const int rem = (w - jb - nb) * nrhs;
        for (int e = tid; e < rem; e += nt) {
            const int i = jb + nb + e / nrhs, r = e % nrhs;
            const T *row = D + (int64_t)i * ld + jb;
            T s = T(0);
            for (int l = 0; l < nb; l++) s += row[l] * y[(jb + l) * nrhs + r];
            y[i * nrhs + r] -= s;
        }
        __syncthreads();
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
__global__ void k_fwd_off(Meta m, const int2 *__restrict__ chunks, const T *__restrict__ coef,
                          T *__restrict__ B, int ldb, int nrhs, int rows_per_chunk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *y = reinterpret_cast<T *>(smem_raw);   // [nrhs][w]
    const int2 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < w * nrhs; e += nt) {
        int r = e / w, j = e - r * w;
        y[e] = B[(int64_t)r * ldb + fc + j];
    }
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const T *P = coef + m.coefoff[c];
    const int rend = min(h, r0 + rows_per_chunk);
    for (int i = r0 + warp; i < rend; i += nw) {
        const T *row = P + (int64_t)i * ld;
        const int grow = m.rowidx[m.rowbase[c] + i];
        for (int r = 0; r < nrhs; r++) {
            T s = T(0);
            for (int j = lane; j < w; j += 32) s += row[j] * y[r * w + j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) atomic_sub(&B[(int64_t)r * ldb + grow], s);
        }
    }
}

// ---------------------------------------------------------------------------
// Backward, off-diagonal gather (kernels/solve_ztrsmsp.c:450
// solve_cblk_ztrsmsp_backward walks browtab): B[fcol+j, :] -= sum_i P[i, j]
// B[row_i, :] over panel rows i >= w of cblk c (P = L for POTRF, U^T for
// GETRF).  Threads along j (coalesced in the row-major panel); a chunk of
// rows per CTA, partial sums combined atomically.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_bwd_off(Meta m, const int2 *__restrict__ chunks, const T *__restrict__ coef,
                          T *__restrict__ B, int ldb, int nrhs, int rows_per_chunk) {
    const int2 ch = chunks[blockIdx.x];
    const int c = ch.x, r0 = ch.y;
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c], h = m.height[c];
    const T *P = coef + m.coefoff[c];
    const int rend = min(h, r0 + rows_per_chunk);
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
        T s[SOLVE_MAXRHS];
        for (int r = 0; r < nrhs; r++) s[r] = T(0);
        for (int i = r0; i < rend; i++) {
            const T pij = P[(int64_t)i * ld + j];
            const int grow = m.rowidx[m.rowbase[c] + i];
            for (int r = 0; r < nrhs; r++) s[r] += pij * B[(int64_t)r * ldb + grow];
        }
        for (int r = 0; r < nrhs; r++) atomic_sub(&B[(int64_t)r * ldb + fc + j], s[r]);
    }
}

// ---------------------------------------------------------------------------
// Backward, diagonal part: B[fcol:fcol+w, :] := D^{-1} B[...] with
// D = L_kk^T (POTRF, Left, Lower, ConjTrans/Trans, NonUnit) or the upper
// triangle U_kk of the LU diagonal block (Left, Upper, NoTrans, NonUnit).
// Blocked by 32 columns from the last block up: warp 0 substitutes through
// the tile, then all threads update the rows above.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_bwd_diag(Meta m, const int *__restrict__ cblks, const T *__restrict__ coefL,
                           T *__restrict__ B, int ldb, int nrhs, int upper) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *x = reinterpret_cast<T *>(smem_raw);   // [w][nrhs]
    const int c = cblks[blockIdx.x];
    const int w = m.width[c], ld = m.ld[c], fc = m.fcol[c];
    const T *D = coefL + m.coefoff[c];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    for (int e = tid; e < w * nrhs; e += nt) {
        int j = e / nrhs, r = e - j * nrhs;
        x[e] = B[(int64_t)r * ldb + fc + j];
    }
    __syncthreads();
    T *tile = x + w * nrhs;                   // [32][33] diagonal tile
    const int nblk = (w + 31) / 32;
    for (int bi = nblk - 1; bi >= 0; bi--) {
        const int jb = bi * 32, nb = min(32, w - jb);
        for (int e = tid; e < nb * nb; e += nt) {
            const int i = e / nb, j = e - i * nb;
            tile[i * 33 + j] = D[(int64_t)(jb + i) * ld + jb + j];
        }
        __syncthreads();
        if (tid < 32) {
            const T dinv = (lane < nb) ? T(1) / tile[lane * 33 + lane] : T(1);
            for (int r = 0; r < nrhs; r++) {
                T v = (lane < nb) ? x[(jb + lane) * nrhs + r] : T(0);
                for (int j = nb - 1; j >= 0; j--) {
                    if (lane == j) v *= dinv;
                    const T xj = __shfl_sync(0xffffffffu, v, j);
                    if (lane < j) {
                        // upper: U[l][j]; Cholesky: L^T[l][j] = L[j][l]
                        const T dlj = upper ? tile[lane * 33 + j] : tile[j * 33 + lane];
                        v -= dlj * xj;
                    }
                }
                if (lane < nb) x[(jb + lane) * nrhs + r] = v;
            }
        }
        __syncthreads();
        const int rem = jb * nrhs;
        for (int e = tid; e < rem; e += nt) {
            const int i = e / nrhs, r = e % nrhs;
            T s = T(0);
            if (upper) {
                const T *row = D + (int64_t)i * ld + jb;
                for (int l = 0; l < nb; l++) s += row[l] * x[(jb + l) * nrhs + r];
            } else {
                for (int l = 0; l < nb; l++) s += D[(int64_t)(jb + l) * ld + i] * x[(jb + l) * nrhs + r];
            }
            x[i * nrhs + r] -= s;
        }
        __syncthreads();
    }
    for (int e = tid; e < w * nrhs; e += nt) {
        int j = e / nrhs, r = e - j * nrhs;
        B[(int64_t)r * ldb + fc + j] = x[e];
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
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t tot = (int64_t)n * nrhs;
    for (; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        int r = (int)(e / n), k = (int)(e - (int64_t)r * n);
        if (!backward) Y[r * ldy + k] = (Tout)X[r * ldx + peritab[k]];
        else Y[r * ldy + peritab[k]] = (Tout)X[r * ldx + k];
    }
}

template <typename Tin, typename Tout>
__global__ void k_convert(int64_t n, const Tin *__restrict__ x, Tout *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] = (Tout)x[i];
}

// ---------------------------------------------------------------------------
// Refinement vector kernels, FP64 (bcsc/bcsc_zspmv.c:629 bcsc_zspmv on the
// permuted matrix held as CSR, one warp per row; bvec_z{dotc,nrm2,axpy,scal,
// copy}, bcsc/bvec_zcompute.c).  Reductions go through per-CTA partials
// finished by one CTA, so results are deterministic.
// ---------------------------------------------------------------------------
__global__ void k_spmv(int n, const int64_t *__restrict__ rowptr, const int *__restrict__ col,
                       const double *__restrict__ val, double alpha, const double *__restrict__ x,
                       double beta, double *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (; row < n; row += nwarps) {
        double s = 0.0;
        for (int64_t k = rowptr[row] + lane; k < rowptr[row + 1]; k += 32) s += val[k] * x[col[k]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) y[row] = alpha * s + (beta == 0.0 ? 0.0 : beta * y[row]);
    }
}

constexpr int RED_THREADS = 256;

__device__ __forceinline__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    if (warp == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// partial[blockIdx] = sum x*y  (or sum x*x when y == nullptr)
__global__ void k_dot_partial(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                              double *__restrict__ partial) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += x[i] * (y ? y[i] : x[i]);
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void k_dot_final(int np, const double *__restrict__ partial, double *__restrict__ out,
                            int do_sqrt) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) *out = do_sqrt ? sqrt(s) : s;
}

__global__ void k_axpy(int64_t n, double alpha, const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}

// p = z + beta * p
__global__ void k_xpby(int64_t n, const double *__restrict__ z, double beta, double *__restrict__ p) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// y += sign * (*alpha) * x with the scalar read from device memory (GMRES
// orthogonalization without a host round trip per projection).
__global__ void k_axpy_dev(int64_t n, const double *__restrict__ alpha, double sign, const double *__restrict__ x,
                           double *__restrict__ y) {
    const double a = sign * (*alpha);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

__global__ void k_scal(int64_t n, double a, double *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] *= a;
}

// x += W(:, 0:k) y  (bvec_zgemv, bcsc/bvec_zcompute.c; W column-major, ld ldw)
__global__ void k_gemv_acc(int64_t n, int k, const double *__restrict__ W, int64_t ldw,
                           const double *__restrict__ y, double *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < k; j++) s += W[i + j * ldw] * y[j];
        x[i] += s;
    }
}

// Gather the permuted-matrix values from the user's values.
__global__ void k_gather_vals(int64_t nnz, const int64_t *__restrict__ src, const double *__restrict__ vals,
                              double *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = vals[src[i]];
}

// Weighted sum of squares for the Frobenius norm (off-diagonal entries of a
// one-triangle symmetric matrix count twice).
__global__ void k_sumsq_partial(int64_t nnz, const double *__restrict__ v, const int8_t *__restrict__ wgt,
                                double *__restrict__ partial) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (int64_t)gridDim.x * blockDim.x)
        s += (double)wgt[i] * v[i] * v[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

}  // namespace pgpu
