// Common definitions of the B200 sopalin kernels: scalar traits, the device
// view of the supernodal structure, and the error-status word.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

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
    const int64_t *invoff; // [cblknbr] offset of the cblk's diagonal-block inverse (TRSM as GEMM), -1 if none
};

// Factorization forms of the kernels (pastix_factotype_t: POTRF = LL^h,
// GETRF = LU, SYTRF = LDL^t, HETRF = LDL^h).  The Hermitian forms (POTRF,
// HETRF) conjugate the transposed operand; for real scalars that is a no-op.
enum FactMode { FM_POTRF = 0, FM_GETRF = 1, FM_SYTRF = 2, FM_HETRF = 3 };
__host__ __device__ constexpr bool fm_conj(int mode) { return mode == FM_POTRF || mode == FM_HETRF; }
__host__ __device__ constexpr bool fm_ldl(int mode) { return mode == FM_SYTRF || mode == FM_HETRF; }

// Elements between the two diagonal-block inverses of an LU cblk (and
// between its L- and U-side TRSM outputs in the scratch): w x ld rounded to 32.
__host__ __device__ inline int64_t inv_span(int64_t rows, int64_t ld) { return (rows * ld + 31) / 32 * 32; }

// Error/status word written by kernels (never traps): bit flags + counters.
struct Status {
    int nbpivots;      // static pivots applied
    int negpivots;     // negative/zero diagonal met in a Cholesky pivot
    int nonfinite;     // NaN/Inf met on a diagonal
    int overflow;      // FP32 down-cast overflow in the mixed fill-in
    int timeout;       // a bounded wait inside a kernel gave up (tile skipped)
    int drain_timeout; // after a time-out, waiting for a CTA's own TMA loads in flight gave up too: the
                       // launch's results are undefined (its shared memory may still receive those bytes)
};

// Complex scalar (interleaved re, im: the layout of pastix_complex64_t /
// pastix_complex32_t and of C99 double/float _Complex).
template <typename R>
struct cplx {
    R re, im;
    cplx() = default;
    __host__ __device__ constexpr cplx(R r, R i = R(0)) : re(r), im(i) {}
    template <typename S>
    __host__ __device__ explicit cplx(const cplx<S> &o) : re(R(o.re)), im(R(o.im)) {}
    __host__ __device__ cplx &operator+=(const cplx &o) { re += o.re; im += o.im; return *this; }
    __host__ __device__ cplx &operator-=(const cplx &o) { re -= o.re; im -= o.im; return *this; }
    __host__ __device__ cplx &operator*=(const cplx &o) {
        const R r = re * o.re - im * o.im;
        im = re * o.im + im * o.re;
        re = r;
        return *this;
    }
};
template <typename R> __host__ __device__ inline cplx<R> operator+(cplx<R> a, const cplx<R> &b) { return a += b; }
template <typename R> __host__ __device__ inline cplx<R> operator-(cplx<R> a, const cplx<R> &b) { return a -= b; }
template <typename R> __host__ __device__ inline cplx<R> operator*(cplx<R> a, const cplx<R> &b) { return a *= b; }
template <typename R> __host__ __device__ inline cplx<R> operator-(const cplx<R> &a) { return cplx<R>(-a.re, -a.im); }
template <typename R> __host__ __device__ inline cplx<R> operator*(R a, const cplx<R> &b) { return cplx<R>(a * b.re, a * b.im); }
// Smith's algorithm for the quotient (scaled by the larger part of b).
template <typename R> __host__ __device__ inline cplx<R> operator/(const cplx<R> &a, const cplx<R> &b) {
    if (fabs(b.re) >= fabs(b.im)) {
        const R r = b.im / b.re, d = b.re + b.im * r;
        return cplx<R>((a.re + a.im * r) / d, (a.im - a.re * r) / d);
    }
    const R r = b.re / b.im, d = b.im + b.re * r;
    return cplx<R>((a.re * r + a.im) / d, (a.im * r - a.re) / d);
}
typedef cplx<float> cfloat;
typedef cplx<double> cdouble;

template <typename T> struct is_cplx { static constexpr bool value = false; };
template <typename R> struct is_cplx<cplx<R>> { static constexpr bool value = true; };

// Real type of a scalar, and the helpers every kernel uses on T.
template <typename T> struct real_of { typedef T type; };
template <typename R> struct real_of<cplx<R>> { typedef R type; };

__host__ __device__ inline float conj_v(float a) { return a; }
__host__ __device__ inline double conj_v(double a) { return a; }
template <typename R> __host__ __device__ inline cplx<R> conj_v(const cplx<R> &a) { return cplx<R>(a.re, -a.im); }
// conjugate when C (Hermitian forms), identity otherwise
template <bool C, typename T> __host__ __device__ inline T cj(const T &a) { return C ? conj_v(a) : a; }

__host__ __device__ inline float real_v(float a) { return a; }
__host__ __device__ inline double real_v(double a) { return a; }
template <typename R> __host__ __device__ inline R real_v(const cplx<R> &a) { return a.re; }

__device__ inline float abs_v(float a) { return fabsf(a); }
__device__ inline double abs_v(double a) { return fabs(a); }
template <typename R> __device__ inline R abs_v(const cplx<R> &a) { return hypot(a.re, a.im); }

__device__ inline float abs2_v(float a) { return a * a; }
__device__ inline double abs2_v(double a) { return a * a; }
template <typename R> __device__ inline R abs2_v(const cplx<R> &a) { return a.re * a.re + a.im * a.im; }

__device__ inline bool finite_v(float a) { return isfinite(a); }
__device__ inline bool finite_v(double a) { return isfinite(a); }
template <typename R> __device__ inline bool finite_v(const cplx<R> &a) { return isfinite(a.re) && isfinite(a.im); }

__device__ inline float sqrt_v(float a) { return sqrtf(a); }
__device__ inline double sqrt_v(double a) { return sqrt(a); }
// Cholesky pivots of a Hermitian matrix are real: the square root of the real part
template <typename R> __device__ inline cplx<R> sqrt_v(const cplx<R> &a) { return cplx<R>(sqrt(a.re), R(0)); }

__device__ __forceinline__ float shfl_v(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ double shfl_v(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <typename R> __device__ __forceinline__ cplx<R> shfl_v(const cplx<R> &v, int src) {
    return cplx<R>(__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src));
}
__device__ __forceinline__ float shfl_xor_v(float v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
__device__ __forceinline__ double shfl_xor_v(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
template <typename R> __device__ __forceinline__ cplx<R> shfl_xor_v(const cplx<R> &v, int m) {
    return cplx<R>(__shfl_xor_sync(0xffffffffu, v.re, m), __shfl_xor_sync(0xffffffffu, v.im, m));
}

__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }
template <typename R> __device__ __forceinline__ void atomic_add(cplx<R> *p, const cplx<R> &v) {
    atomicAdd(&p->re, v.re);
    atomicAdd(&p->im, v.im);
}
__device__ __forceinline__ void atomic_sub(double *p, double v) { atomicAdd(p, -v); }
__device__ __forceinline__ void atomic_sub(float *p, float v) { atomicAdd(p, -v); }
template <typename R> __device__ __forceinline__ void atomic_sub(cplx<R> *p, const cplx<R> &v) {
    atomicAdd(&p->re, -v.re);
    atomicAdd(&p->im, -v.im);
}

// Task timing for the learned cost model: when prof != nullptr, thread 0 of
// each CTA stores the global timer (ns) at the CTA's start and end in
// prof[2 * blockIdx.x + {0, 1}].
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Block-cooperative copy of `total` elements, element e read by src(e) and
// written by dst(e, v), U loads in flight per thread: the loads of a batch
// are issued before any of their stores, so a global -> shared staging loop
// costs one memory latency per U elements instead of one per element.
template <int U = 8, typename Src, typename Dst>
__device__ __forceinline__ void batched_copy(int total, int tid, int nt, Src src, Dst dst) {
    for (int e0 = tid; e0 < total; e0 += nt * U) {
        decltype(src(0)) r[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = e0 + u * nt;
            if (e < total) r[u] = src(e);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = e0 + u * nt;
            if (e < total) dst(e, r[u]);
        }
    }
}

// Round to TF32 (nearest, ties away from zero): the "hi" part of a 3xTF32
// operand split x = hi + lo.
__device__ __forceinline__ float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Shared-memory address and asynchronous global -> shared copies
// (cp.async: 16 bytes through L2 only, or 4 / 8 / 16 bytes through L1; a
// commit closes a group, wait<N> leaves at most N groups in flight).
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// mbarriers (shared::cta) and bulk asynchronous copies global -> shared.
__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

// Bounded wait on an mbarrier phase; false on time-out (about 2 s).
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 4000000000LL) return false;
    }
}
__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t addr, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes) : "memory");
}

// Bulk asynchronous copy of `bytes` (a multiple of 16; both addresses 16-byte
// aligned) from global memory into this CTA's shared memory, completing on
// mbar (complete_tx).  No multicast.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void *gptr, bool valid) {
    const int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(gptr), "r"(sz) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_ca(uint32_t saddr, const void *gptr) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(saddr), "l"(gptr), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

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
