// Common definitions of the B200 sopalin kernels: scalar traits, the device
// view of the supernodal structure, and the error-status word.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace pgpu {

// ---------------------------------------------------------------------------
// Device view of the SolverMatrix (blend/solver.h:137-273) in the layout the
// kernels use.  Every cblk c owns a row-major panel of h_c rows and ld_c
// columns (the first w_c are used) starting at coefoff[c]; row i of the panel
// is the global (permuted) row rowidx[rowbase[c] + i].  The diagonal block
// occupies rows [0, w_c), off-diagonal block b occupies rows
// [rowoff[b], rowoff[b] + m_b).  Row-major panels make every operand of the
// update GEMM K-major (K = w_c contiguous) and every panel row an independent
// triangular solve.
// ---------------------------------------------------------------------------
struct Meta {
    int n;
    int cblknbr;
    int bloknbr;
    const int *fcol;       // [cblknbr] first column
    const int *width;      // [cblknbr] w_c
    const int *height;     // [cblknbr] h_c (stride)
    const int *ld;         // [cblknbr] panel leading dimension (>= w_c)
    const int64_t *coefoff;// [cblknbr] panel offset (elements)
    const int *fblok;      // [cblknbr+1] first blok (the diagonal one)
    const int64_t *rowbase;// [cblknbr] offset in rowidx
    const int *rowidx;     // [sum h_c] global row of each panel row
    const int *bfrow;      // [bloknbr] frownum
    const int *blrow;      // [bloknbr] lrownum
    const int *browoff;    // [bloknbr] first panel row of the block
    const int *bfcblk;     // [bloknbr] facing cblk
};

// Error/status word written by kernels (never traps): bit flags + counters.
struct Status {
    int nbpivots;      // static pivots applied
    int negpivots;     // negative/zero diagonal met in a Cholesky pivot
    int nonfinite;     // NaN/Inf met on a diagonal
    int overflow;      // FP32 down-cast overflow in the mixed fill-in
    int timeout;       // a bounded wait inside a kernel gave up (tile skipped)
};

template <typename T> struct ScalarOps;
template <> struct ScalarOps<double> {
    static __device__ __forceinline__ double absval(double a) { return fabs(a); }
    static __device__ __forceinline__ double sqrtv(double a) { return sqrt(a); }
};
template <> struct ScalarOps<float> {
    static __device__ __forceinline__ float absval(float a) { return fabsf(a); }
    static __device__ __forceinline__ float sqrtv(float a) { return sqrtf(a); }
};

__device__ __forceinline__ void atomic_sub(double *p, double v) { atomicAdd(p, -v); }
__device__ __forceinline__ void atomic_sub(float *p, float v) { atomicAdd(p, -v); }

// Panel row of global row r inside cblk f: binary search over f's blocks
// (sorted by frownum, blend/solver.h:497-514 is_block_inside_fblock walks
// them linearly).  Returns -1 if r is not a row of f.
__device__ __forceinline__ int panel_row_of(const Meta &m, int f, int r) {
    int lo = m.fblok[f], hi = m.fblok[f + 1] - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (m.bfrow[mid] <= r) lo = mid; else hi = mid - 1;
    }
    if (r < m.bfrow[lo] || r > m.blrow[lo]) return -1;
    return m.browoff[lo] + (r - m.bfrow[lo]);
}

}  // namespace pgpu
