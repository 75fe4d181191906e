// Host side of the B200 sopalin replacement: the C ABI declared in
// include/pastix_gpu.h, the device layout of the coeftab, the level schedule
// and the drivers of numfact / solve / refinement.
#include "pastix_gpu.h"
#include "pgpu_factor.cuh"
#include "pgpu_solve.cuh"
#include "pgpu_panel.cuh"
#include "pgpu_gemm_tc.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

using namespace pgpu;

#define PGPU_CHECK(x)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "pastix_gpu: %s failed: %s (%s:%d)\n", #x,                 \
                    cudaGetErrorString(e_), __FILE__, __LINE__);                       \
            return e_ == cudaErrorMemoryAllocation ? PASTIX_GPU_ERR_OUTOFMEMORY        \
                                                   : PASTIX_GPU_ERR_INTERNAL;          \
        }                                                                              \
    } while (0)

namespace {

template <typename T>
struct DArr {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t cnt) {
        release();
        n = cnt;
        if (!cnt) return cudaSuccess;
        return cudaMalloc(&p, cnt * sizeof(T));
    }
    cudaError_t upload(const std::vector<T> &v, cudaStream_t s) {
        cudaError_t e = alloc(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    DArr() = default;
    DArr(const DArr &) = delete;
    DArr &operator=(const DArr &) = delete;
    ~DArr() { release(); }
};

inline int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }
inline int cdiv(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

const int SOLVE_ROWS_PER_CHUNK = 32;

bool is_device_ptr(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace

struct pastix_gpu_s {
    int device = 0;
    int64_t iparm[PGPU_IPARM_SIZE];
    double dparm[PGPU_DPARM_SIZE];
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6];

    // ---- structure (host copies) ----
    int n = 0, cblknbr = 0, bloknbr = 0;
    std::vector<int> fcol, width, height, ld, fblok, bfrow, blrow, browoff, bfcblk, rowidx, col2cblk;
    std::vector<int64_t> coefoff, rowbase;
    std::vector<int> peritab;
    int64_t coefnbr = 0;      // elements of one (L or U) coeftab incl. padding
    int maxw = 0;
    int nlevels = 0;
    std::vector<int> lvl_ptr, lvl_cblks, lvl_maxw;
    double thflops_potrf = 0, thflops_getrf = 0;

    // ---- device structure ----
    DArr<int> d_fcol, d_width, d_height, d_ld, d_fblok, d_rowidx, d_bfrow, d_blrow, d_browoff, d_bfcblk,
        d_lvl_cblks, d_peritab;
    DArr<int64_t> d_coefoff, d_rowbase;
    Meta meta{};

    // ---- factorization plan (per factotype) ----
    int plan_fact = -1;
    std::vector<int> tile_ptr, tctile_ptr, trsm_ptr, lvl_plrows, lvl_porows;
    DArr<int4> d_tiles, d_tctiles, d_trsm;
    double tc_flops = 0;   // update-GEMM flops on the tensor-core path
    DArr<GemmTask> d_tasks;
    std::vector<int> solve_ptr;
    DArr<int2> d_solve_chunks;

    // ---- matrix ----
    int mtxtype = PGPU_SYMMETRIC, flttype = PGPU_DOUBLE;
    int64_t nnz = 0;
    DArr<int64_t> d_fill_dst;   // per user nnz: coeftab offset (U entries offset by coefnbr)
    DArr<int8_t> d_wgt;         // Frobenius weight per user nnz
    DArr<int64_t> d_csr_ptr, d_csr_src;
    DArr<int> d_csr_col;
    DArr<double> d_csr_val, d_vals;
    bool have_spm = false;

    // ---- numerical state ----
    DArr<unsigned char> d_coef;
    int coef_float = 0;     // factor precision of d_coef
    int fact_done = -1;     // factotype of the factors in d_coef, -1 if none
    DArr<Status> d_status;
    DArr<double> d_partial, d_scalar;
    DArr<unsigned char> d_work;   // solve workspace (n x 16 in factor precision)
    DArr<double> d_rhs, d_x, d_r, d_z, d_p, d_ap, d_gm;   // refinement vectors
    DArr<double> d_sr_b, d_sr_x;   // solve_and_refine staging of host B / X
    DArr<double> d_gmV, d_gmW, d_gmh;   // GMRES basis, preconditioned basis, projections
    std::vector<cudaEvent_t> evpool;   // per-launch timing events
    double gemm_flops[5] = {0};        // update-GEMM flops per factotype
    double stats[16] = {0};
};

// --------------------------------------------------------------------------
static void default_params(int64_t *iparm, double *dparm) {
    // common/api.c:411-560 defaults for the entries this layer reads
    std::fill(iparm, iparm + PGPU_IPARM_SIZE, 0);
    std::fill(dparm, dparm + PGPU_DPARM_SIZE, 0.0);
    iparm[PGPU_IPARM_FACTORIZATION] = PGPU_FACT_GETRF;
    iparm[PGPU_IPARM_REFINEMENT] = PGPU_REFINE_GMRES;
    iparm[PGPU_IPARM_ITERMAX] = 250;
    iparm[PGPU_IPARM_GMRES_IM] = 25;
    dparm[PGPU_DPARM_EPSILON_REFINEMENT] = -1.0;
    dparm[PGPU_DPARM_EPSILON_MAGN_CTRL] = 0.0;
}

extern "C" int pastix_gpu_init(pastix_gpu_t **pctx, int device, const int64_t *iparm, const double *dparm) {
    if (!pctx) return PASTIX_GPU_ERR_BADPARAMETER;
    *pctx = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        fprintf(stderr, "pastix_gpu: no CUDA device available\n");
        return PASTIX_GPU_ERR_INTERNAL;
    }
    if (device < 0 || device >= ndev) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(device));
    pastix_gpu_t *ctx = new pastix_gpu_t();
    ctx->device = device;
    default_params(ctx->iparm, ctx->dparm);
    if (iparm) std::memcpy(ctx->iparm, iparm, sizeof(ctx->iparm));
    if (dparm) std::memcpy(ctx->dparm, dparm, sizeof(ctx->dparm));
    PGPU_CHECK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    for (auto &e : ctx->ev) PGPU_CHECK(cudaEventCreate(&e));
    PGPU_CHECK(ctx->d_status.alloc(1));
    PGPU_CHECK(ctx->d_partial.alloc(1024));
    PGPU_CHECK(ctx->d_scalar.alloc(16));
    *pctx = ctx;
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// Structure handoff: device layout + level schedule.
// --------------------------------------------------------------------------
extern "C" int pastix_gpu_structure(pastix_gpu_t *ctx, int64_t n, int64_t cblknbr, const int64_t *cblktab,
                                    int64_t bloknbr, const int64_t *bloktab, int64_t brownbr,
                                    const int64_t *browtab, const int64_t *permtab, const int64_t *peritab) {
    (void)brownbr; (void)browtab; (void)permtab;
    if (!ctx || n <= 0 || cblknbr <= 0 || !cblktab || !bloktab || !peritab) return PASTIX_GPU_ERR_BADPARAMETER;
    if (n > INT32_MAX || bloknbr > INT32_MAX) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(ctx->device));
    auto &C = *ctx;
    C.n = (int)n;
    C.cblknbr = (int)cblknbr;
    C.bloknbr = (int)bloknbr;
    const int nc = C.cblknbr, nb = C.bloknbr;
    C.fcol.resize(nc); C.width.resize(nc); C.height.resize(nc); C.ld.resize(nc);
    C.coefoff.resize(nc); C.rowbase.resize(nc); C.fblok.resize(nc + 1);
    C.bfrow.resize(nb); C.blrow.resize(nb); C.browoff.resize(nb); C.bfcblk.resize(nb);
    C.col2cblk.assign(n, -1);
    C.rowidx.clear();
    for (int b = 0; b < nb; b++) {
        C.bfrow[b] = (int)bloktab[4 * b + 0];
        C.blrow[b] = (int)bloktab[4 * b + 1];
        C.bfcblk[b] = (int)bloktab[4 * b + 3];
    }
    int64_t off = 0;
    C.maxw = 0;
    for (int c = 0; c <= nc; c++) C.fblok[c] = (int)cblktab[4 * c + 2];
    if (C.fblok[nc] != nb) return PASTIX_GPU_ERR_BADPARAMETER;
    double fl_potrf = 0, fl_getrf = 0;
    for (int c = 0; c < nc; c++) {
        const int fc = (int)cblktab[4 * c + 0], lc = (int)cblktab[4 * c + 1];
        const int w = lc - fc + 1;
        const int b0 = C.fblok[c], b1 = C.fblok[c + 1];
        if (w <= 0 || b1 <= b0 || C.bfrow[b0] != fc || C.blrow[b0] != lc) return PASTIX_GPU_ERR_BADPARAMETER;
        C.fcol[c] = fc;
        C.width[c] = w;
        C.maxw = std::max(C.maxw, w);
        for (int j = fc; j <= lc; j++) C.col2cblk[j] = c;
        C.rowbase[c] = (int64_t)C.rowidx.size();
        int h = 0;
        for (int b = b0; b < b1; b++) {
            if (C.blrow[b] < C.bfrow[b] || C.blrow[b] >= n) return PASTIX_GPU_ERR_BADPARAMETER;
            if (b > b0 && (C.bfcblk[b] <= c || C.bfcblk[b] >= nc || C.bfrow[b] <= C.blrow[b - 1]))
                return PASTIX_GPU_ERR_BADPARAMETER;
            C.browoff[b] = h;
            for (int r = C.bfrow[b]; r <= C.blrow[b]; r++) C.rowidx.push_back(r);
            h += C.blrow[b] - C.bfrow[b] + 1;
        }
        C.height[c] = h;
        C.ld[c] = (int)round_up(w, 4);
        C.coefoff[c] = off;
        off += round_up((int64_t)h * C.ld[c], 32);
        // algorithmic flops (common/flops.h: FLOPS_DPOTRF / DGETRF, DTRSM, DGEMM)
        const double W = w, M = h - w;
        fl_potrf += W * W * W / 3.0 + W * W / 2.0 + W / 6.0 + M * W * W;
        fl_getrf += 2.0 * W * W * W / 3.0 - W * W / 2.0 + 5.0 * W / 6.0 + 2.0 * M * W * W;
        for (int b = b0 + 1; b < b1; b++) {
            const double N = C.blrow[b] - C.bfrow[b] + 1, Mb = h - C.browoff[b];
            fl_potrf += 2.0 * Mb * N * W;
            fl_getrf += 2.0 * Mb * N * W + (b + 1 < b1 ? 2.0 * (Mb - N) * N * W : 0.0);
        }
    }
    // every block must lie inside the columns of the cblk it faces, which is
    // what lets the update GEMM address its target column directly
    for (int b = 0; b < nb; b++) {
        const int f = C.bfcblk[b];
        if (f < 0 || f >= nc || C.bfrow[b] < C.fcol[f] || C.blrow[b] > C.fcol[f] + C.width[f] - 1)
            return PASTIX_GPU_ERR_BADPARAMETER;
    }
    // the panel TRSM keeps TRSM_ROWS x w elements in shared memory
    if (C.maxw > 400) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    C.thflops_potrf = fl_potrf;
    C.thflops_getrf = fl_getrf;
    for (int j = 0; j < n; j++)
        if (C.col2cblk[j] < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    C.coefnbr = off;
    C.peritab.assign(peritab, peritab + n);

    // level schedule: level(c) = 1 + max level of the cblks whose first
    // off-diagonal block faces c (elimination-tree children)
    std::vector<int> level(nc, 0);
    for (int c = 0; c < nc; c++) {
        if (C.fblok[c + 1] - C.fblok[c] > 1) {
            int p = C.bfcblk[C.fblok[c] + 1];
            level[p] = std::max(level[p], level[c] + 1);
        }
    }
    C.nlevels = 0;
    for (int c = 0; c < nc; c++) C.nlevels = std::max(C.nlevels, level[c] + 1);
    C.lvl_ptr.assign(C.nlevels + 1, 0);
    for (int c = 0; c < nc; c++) C.lvl_ptr[level[c] + 1]++;
    for (int l = 0; l < C.nlevels; l++) C.lvl_ptr[l + 1] += C.lvl_ptr[l];
    C.lvl_cblks.assign(nc, 0);
    C.lvl_maxw.assign(C.nlevels, 0);
    {
        std::vector<int> pos(C.lvl_ptr.begin(), C.lvl_ptr.end() - 1);
        for (int c = 0; c < nc; c++) {
            C.lvl_cblks[pos[level[c]]++] = c;
            C.lvl_maxw[level[c]] = std::max(C.lvl_maxw[level[c]], C.width[c]);
        }
    }

    // device copies
    cudaStream_t s = C.stream;
    PGPU_CHECK(C.d_fcol.upload(C.fcol, s));
    PGPU_CHECK(C.d_width.upload(C.width, s));
    PGPU_CHECK(C.d_height.upload(C.height, s));
    PGPU_CHECK(C.d_ld.upload(C.ld, s));
    PGPU_CHECK(C.d_coefoff.upload(C.coefoff, s));
    PGPU_CHECK(C.d_fblok.upload(C.fblok, s));
    PGPU_CHECK(C.d_rowbase.upload(C.rowbase, s));
    PGPU_CHECK(C.d_rowidx.upload(C.rowidx, s));
    PGPU_CHECK(C.d_bfrow.upload(C.bfrow, s));
    PGPU_CHECK(C.d_blrow.upload(C.blrow, s));
    PGPU_CHECK(C.d_browoff.upload(C.browoff, s));
    PGPU_CHECK(C.d_bfcblk.upload(C.bfcblk, s));
    PGPU_CHECK(C.d_lvl_cblks.upload(C.lvl_cblks, s));
    PGPU_CHECK(C.d_peritab.upload(C.peritab, s));
    C.meta = Meta{C.n, nc, nb, C.d_fcol.p, C.d_width.p, C.d_height.p, C.d_ld.p, C.d_coefoff.p,
                  C.d_fblok.p, C.d_rowbase.p, C.d_rowidx.p, C.d_bfrow.p, C.d_blrow.p, C.d_browoff.p,
                  C.d_bfcblk.p};

    // solve chunks (independent of the factorization type)
    std::vector<int2> sch;
    C.solve_ptr.assign(C.nlevels + 1, 0);
    for (int l = 0; l < C.nlevels; l++) {
        for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1]; q++) {
            int c = C.lvl_cblks[q];
            for (int r0 = C.width[c]; r0 < C.height[c]; r0 += SOLVE_ROWS_PER_CHUNK) sch.push_back(make_int2(c, r0));
        }
        C.solve_ptr[l + 1] = (int)sch.size();
    }
    PGPU_CHECK(C.d_solve_chunks.upload(sch, s));
    C.plan_fact = -1;
    C.fact_done = -1;
    C.d_coef.release();
    PGPU_CHECK(cudaStreamSynchronize(s));
    return PASTIX_GPU_SUCCESS;
}

// Panel row of global row r in cblk c (host mirror of panel_row_of).
static int host_panel_row(const pastix_gpu_t &C, int c, int r) {
    int lo = C.fblok[c], hi = C.fblok[c + 1] - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (C.bfrow[mid] <= r) lo = mid; else hi = mid - 1;
    }
    if (r < C.bfrow[lo] || r > C.blrow[lo]) return -1;
    return C.browoff[lo] + (r - C.bfrow[lo]);
}

// --------------------------------------------------------------------------
// Pattern handoff: fill-in map (bcsc -> coeftab) and the permuted CSR.
// --------------------------------------------------------------------------
extern "C" int pastix_gpu_spm(pastix_gpu_t *ctx, int mtxtype, int flttype, int64_t n, const int64_t *colptr,
                              const int64_t *rowptr) {
    if (!ctx || !colptr || !rowptr) return PASTIX_GPU_ERR_BADPARAMETER;
    if (n != ctx->n) return PASTIX_GPU_ERR_BADPARAMETER;
    if (flttype != PGPU_DOUBLE) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    if (mtxtype != PGPU_GENERAL && mtxtype != PGPU_SYMMETRIC && mtxtype != PGPU_HERMITIAN)
        return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(ctx->device));
    auto &C = *ctx;
    C.mtxtype = mtxtype;
    C.flttype = flttype;
    const int64_t nnz = colptr[n];
    C.nnz = nnz;
    std::vector<int> perm(n);
    for (int k = 0; k < n; k++) perm[C.peritab[k]] = k;
    std::vector<int64_t> dst(nnz);
    std::vector<int8_t> wgt(nnz);
    const bool sym = (mtxtype != PGPU_GENERAL);
    // permuted full matrix as (row, col, src) triplets
    std::vector<int64_t> rcount(n + 1, 0);
    for (int64_t j = 0; j < n; j++) {
        for (int64_t k = colptr[j]; k < colptr[j + 1]; k++) {
            int64_t i = rowptr[k];
            if (i < 0 || i >= n) return PASTIX_GPU_ERR_BADPARAMETER;
            int pi = perm[i], pj = perm[j];
            wgt[k] = (sym && i != j) ? 2 : 1;
            rcount[pi + 1]++;
            if (sym && i != j) rcount[pj + 1]++;
            if (sym && pi < pj) std::swap(pi, pj);
            int64_t d;
            if (pi >= pj) {
                int c = C.col2cblk[pj];
                int pr = host_panel_row(C, c, pi);
                if (pr < 0) return PASTIX_GPU_ERR_BADPARAMETER;
                d = C.coefoff[c] + (int64_t)pr * C.ld[c] + (pj - C.fcol[c]);
            } else {
                // general, upper entry A(pi, pj), pi < pj
                int c = C.col2cblk[pi];
                if (C.col2cblk[pj] == c) {
                    // inside the diagonal block: kept in L's square
                    d = C.coefoff[c] + (int64_t)(pi - C.fcol[c]) * C.ld[c] + (pj - C.fcol[c]);
                } else {
                    int pr = host_panel_row(C, c, pj);
                    if (pr < 0) return PASTIX_GPU_ERR_BADPARAMETER;
                    d = C.coefnbr + C.coefoff[c] + (int64_t)pr * C.ld[c] + (pi - C.fcol[c]);
                }
            }
            dst[k] = d;
        }
    }
    for (int64_t i = 0; i < n; i++) rcount[i + 1] += rcount[i];
    const int64_t fnnz = rcount[n];
    std::vector<int> ccol(fnnz);
    std::vector<int64_t> csrc(fnnz);
    {
        std::vector<int64_t> pos(rcount.begin(), rcount.end() - 1);
        for (int64_t j = 0; j < n; j++) {
            for (int64_t k = colptr[j]; k < colptr[j + 1]; k++) {
                int64_t i = rowptr[k];
                int pi = perm[i], pj = perm[j];
                int64_t q = pos[pi]++;
                ccol[q] = pj;
                csrc[q] = k;
                if (sym && i != j) {
                    q = pos[pj]++;
                    ccol[q] = pi;
                    csrc[q] = k;
                }
            }
        }
    }
    cudaStream_t s = C.stream;
    PGPU_CHECK(C.d_fill_dst.upload(dst, s));
    PGPU_CHECK(C.d_wgt.upload(wgt, s));
    PGPU_CHECK(C.d_csr_ptr.upload(rcount, s));
    PGPU_CHECK(C.d_csr_col.upload(ccol, s));
    PGPU_CHECK(C.d_csr_src.upload(csrc, s));
    PGPU_CHECK(C.d_csr_val.alloc(fnnz));
    PGPU_CHECK(C.d_vals.alloc(nnz));
    PGPU_CHECK(cudaStreamSynchronize(s));
    C.have_spm = true;
    C.fact_done = -1;
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// Factorization plan for one factorization type.
// --------------------------------------------------------------------------
// Off-diagonal rows of cblks taller than fuse_rows are solved by
// k_trsm_rows; shorter panels are factorized whole by k_panel_factor.
static int fuse_rows_for(bool lu, bool fp32) {
    if (lu) return fp32 ? 256 : 96;
    return fp32 ? 1024 : 512;
}
static const int TRSM_TR = 32;   // panel rows per k_trsm_rows CTA

// Single-precision update GEMMs large enough for a 128 x 128 tensor-core tile
// go to k_gemm_scatter_tc.  PASTIX_GPU_MIXED_GEMM selects the operand mode:
// "3xtf32" (default; split products, about FP32 accuracy), "tf32" (one TF32
// product) or "fp32" (no tensor cores: FP32 FMA tiles only).
enum { MG_FP32 = 0, MG_TF32 = 1, MG_3XTF32 = 2 };
static int mixed_gemm_mode() {
    const char *e = getenv("PASTIX_GPU_MIXED_GEMM");
    if (e && std::strcmp(e, "fp32") == 0) return MG_FP32;
    if (e && std::strcmp(e, "tf32") == 0) return MG_TF32;
    return MG_3XTF32;
}
static bool tc_enabled() { return mixed_gemm_mode() != MG_FP32; }
static bool tc_task(int M, int N, int K) { return K >= 32 && M >= 64 && N >= 32 && (int64_t)M * N >= 128 * 64; }

static int build_fact_plan(pastix_gpu_t &C, int fact, bool fp32) {
    const bool use_tc = fp32 && tc_enabled();
    const int key = fact * 4 + (fp32 ? 1 : 0) + (use_tc ? 2 : 0);
    if (C.plan_fact == key) return PASTIX_GPU_SUCCESS;
    const bool lu = (fact == PGPU_FACT_GETRF);
    const int fuse = fuse_rows_for(lu, fp32);
    std::vector<int4> tiles, trsm, tctiles;
    std::vector<GemmTask> tasks;
    double gflops = 0, tcflops = 0;
    C.tile_ptr.assign(C.nlevels + 1, 0);
    C.tctile_ptr.assign(C.nlevels + 1, 0);
    C.trsm_ptr.assign(C.nlevels + 1, 0);
    C.lvl_plrows.assign(C.nlevels, 0);
    C.lvl_porows.assign(C.nlevels, 0);
    for (int l = 0; l < C.nlevels; l++) {
        for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1]; q++) {
            const int c = C.lvl_cblks[q];
            const int w = C.width[c], h = C.height[c];
            const int rows = (h <= fuse) ? h : w;
            C.lvl_plrows[l] = std::max(C.lvl_plrows[l], rows);
            C.lvl_porows[l] = std::max(C.lvl_porows[l], rows - w);
            if (h > fuse)
                for (int r0 = w; r0 < h; r0 += TRSM_TR) {
                    trsm.push_back(make_int4(c, r0, 0, lu ? 1 : 0));
                    if (lu) trsm.push_back(make_int4(c, r0, 1, 2));
                }
            const int b1 = C.fblok[c + 1];
            for (int b = C.fblok[c] + 1; b < b1; b++) {
                const int f = C.bfcblk[b];
                const int N = C.blrow[b] - C.bfrow[b] + 1;
                auto add = [&](int arow0, int flags) {
                    const int M = h - arow0;
                    if (M <= 0) return;
                    const int id = (int)tasks.size();
                    tasks.push_back(GemmTask{c, b, f, arow0, M, flags});
                    gflops += 2.0 * M * N * w;
                    if (use_tc && tc_task(M, N, w)) {
                        tcflops += 2.0 * M * N * w;
                        for (int tm = 0; tm < cdiv(M, TC_BM); tm++)
                            for (int tn = 0; tn < cdiv(N, TC_BN); tn++) {
                                if ((flags & 8) && tm < tn) continue;
                                tctiles.push_back(make_int4(id, tm, tn, 0));
                            }
                        return;
                    }
                    for (int tm = 0; tm < cdiv(M, GEMM_TM); tm++)
                        for (int tn = 0; tn < cdiv(N, GEMM_TN); tn++) {
                            if ((flags & 8) && tm < tn) continue;   // strictly upper tiles of the diagonal block
                            tiles.push_back(make_int4(id, tm, tn, 0));
                        }
                };
                if (!lu) {
                    add(C.browoff[b], 8);
                } else {
                    add(C.browoff[b], 2);                          // L side: A = L, B = U^T rows of b
                    if (b + 1 < b1) add(C.browoff[b + 1], 1 | 4);  // U side: A = U^T, B = L rows of b
                }
            }
        }
        C.tile_ptr[l + 1] = (int)tiles.size();
        C.tctile_ptr[l + 1] = (int)tctiles.size();
        C.trsm_ptr[l + 1] = (int)trsm.size();
    }
    cudaStream_t s = C.stream;
    PGPU_CHECK(C.d_tiles.upload(tiles, s));
    PGPU_CHECK(C.d_tctiles.upload(tctiles, s));
    PGPU_CHECK(C.d_trsm.upload(trsm, s));
    PGPU_CHECK(C.d_tasks.upload(tasks, s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    C.plan_fact = key;
    C.gemm_flops[fact] = gflops;
    C.tc_flops = tcflops;
    return PASTIX_GPU_SUCCESS;
}

static const int SMEM_LIMIT = 227 * 1024;

// Per-launch timing: one event recorded before every launch (and one after
// the last), so launch i took ev[i+1] - ev[i]; kinds[i] says which phase.
struct LaunchTimer {
    pastix_gpu_t &C;
    std::vector<int> kinds;
    int used = 0;
    explicit LaunchTimer(pastix_gpu_t &c) : C(c) {}
    cudaError_t mark(int kind) {
        if (used >= (int)C.evpool.size()) {
            cudaEvent_t e;
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return r;
            C.evpool.push_back(e);
        }
        kinds.push_back(kind);
        return cudaEventRecord(C.evpool[used++], C.stream);
    }
    // after the stream was synchronized: accumulate ms per kind
    void collect(double *ms, int nkind) {
        for (int k = 0; k < nkind; k++) ms[k] = 0;
        for (int i = 0; i + 1 < used; i++) {
            float t = 0;
            if (kinds[i] >= 0 && kinds[i] < nkind && cudaEventElapsedTime(&t, C.evpool[i], C.evpool[i + 1]) == cudaSuccess)
                ms[kinds[i]] += t;
        }
    }
};

enum { PH_DIAG = 0, PH_TRSM = 1, PH_GEMM = 2, PH_TC = 3, PH_END = 4 };

template <typename T>
static int run_factor(pastix_gpu_t &C, int fact, double crit, int *launches, LaunchTimer &tm) {
    const bool lu = (fact == PGPU_FACT_GETRF);
    T *coefL = reinterpret_cast<T *>(C.d_coef.p);
    T *coefU = lu ? coefL + C.coefnbr : coefL;
    cudaStream_t s = C.stream;
    const int fuse = fuse_rows_for(lu, sizeof(T) == 4);
    auto kpanel = lu ? k_panel_factor<T, true> : k_panel_factor<T, false>;
    PGPU_CHECK(cudaFuncSetAttribute(kpanel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(k_trsm_rows<T, TRSM_TR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    SMEM_LIMIT));
    const bool split = (mixed_gemm_mode() == MG_3XTF32);
    if constexpr (sizeof(T) == 4) {
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tc_smem_bytes<false>()));
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tc_smem_bytes<true>()));
    }
    int nl = 0, ngemm = 0;
    for (int l = 0; l < C.nlevels; l++) {
        const int ncb = C.lvl_ptr[l + 1] - C.lvl_ptr[l];
        const int mw = C.lvl_maxw[l];
        const int pl = C.lvl_plrows[l], pu = lu ? mw : 0, po = lu ? C.lvl_porows[l] : 0;
        const size_t psm = (size_t)(PB * PBL + (size_t)(pl + pu + po) * PBL) * sizeof(T);
        if (psm > (size_t)SMEM_LIMIT) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
        PGPU_CHECK(tm.mark(PH_DIAG));
        kpanel<<<ncb, 256, psm, s>>>(C.meta, C.d_lvl_cblks.p + C.lvl_ptr[l], coefL, coefU, crit, fuse, pl, pu,
                                     C.d_status.p);
        nl++;
        const int ntr = C.trsm_ptr[l + 1] - C.trsm_ptr[l];
        if (ntr) {
            const size_t tsm = ((size_t)TRSM_TR * (mw + 1) + PB * PBL + (size_t)mw * PBL) * sizeof(T);
            if (tsm > (size_t)SMEM_LIMIT) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
            PGPU_CHECK(tm.mark(PH_TRSM));
            k_trsm_rows<T, TRSM_TR><<<ntr, 256, tsm, s>>>(C.meta, C.d_trsm.p + C.trsm_ptr[l], coefL, coefU, mw);
            nl++;
        }
        const int nti = C.tile_ptr[l + 1] - C.tile_ptr[l];
        if (nti) {
            PGPU_CHECK(tm.mark(PH_GEMM));
            k_gemm_scatter<T><<<nti, 256, 0, s>>>(C.meta, C.d_tiles.p + C.tile_ptr[l], C.d_tasks.p, coefL, coefU);
            nl++;
            ngemm++;
        }
        if constexpr (sizeof(T) == 4) {
            const int ntc = C.tctile_ptr[l + 1] - C.tctile_ptr[l];
            if (ntc) {
                PGPU_CHECK(tm.mark(PH_TC));
                if (split)
                    k_gemm_scatter_tc<true><<<ntc, TC_THREADS, tc_smem_bytes<true>(), s>>>(
                        C.meta, C.d_tctiles.p + C.tctile_ptr[l], C.d_tasks.p, coefL, coefU, C.d_status.p);
                else
                    k_gemm_scatter_tc<false><<<ntc, TC_THREADS, tc_smem_bytes<false>(), s>>>(
                        C.meta, C.d_tctiles.p + C.tctile_ptr[l], C.d_tasks.p, coefL, coefU, C.d_status.p);
                nl++;
                ngemm++;
            }
        }
    }
    PGPU_CHECK(tm.mark(PH_END));
    PGPU_CHECK(cudaGetLastError());
    *launches = nl;
    C.stats[7] = ngemm;
    return PASTIX_GPU_SUCCESS;
}

static int dev_norm_frob(pastix_gpu_t &C, double *out) {
    cudaStream_t s = C.stream;
    const int nb = 512;
    k_sumsq_partial<<<nb, RED_THREADS, 0, s>>>(C.nnz, C.d_vals.p, C.d_wgt.p, C.d_partial.p);
    k_dot_final<<<1, RED_THREADS, 0, s>>>(nb, C.d_partial.p, C.d_scalar.p, 1);
    PGPU_CHECK(cudaMemcpyAsync(out, C.d_scalar.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_numfact(pastix_gpu_t *ctx, const void *values) {
    if (!ctx || !values) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (!C.have_spm || C.cblknbr == 0) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(C.device));
    const int fact = (int)C.iparm[PGPU_IPARM_FACTORIZATION];
    if (fact != PGPU_FACT_POTRF && fact != PGPU_FACT_GETRF) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    if (fact == PGPU_FACT_POTRF && C.mtxtype == PGPU_GENERAL) return PASTIX_GPU_ERR_BADPARAMETER;
    const int mixed = C.iparm[PGPU_IPARM_MIXED] ? 1 : 0;
    int rc = build_fact_plan(C, fact, mixed != 0);
    if (rc) return rc;
    const size_t esz = mixed ? sizeof(float) : sizeof(double);
    const size_t ncoef = (size_t)C.coefnbr * (fact == PGPU_FACT_GETRF ? 2 : 1);
    if (C.d_coef.n < ncoef * esz) {
        C.d_coef.release();
        PGPU_CHECK(C.d_coef.alloc(ncoef * esz));
    }
    cudaStream_t s = C.stream;
    PGPU_CHECK(cudaEventRecord(C.ev[0], s));
    // values in (pastix_subtask_spm2bcsc), norm, bcsc -> coeftab
    if (is_device_ptr(values))
        PGPU_CHECK(cudaMemcpyAsync(C.d_vals.p, values, C.nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    else
        PGPU_CHECK(cudaMemcpyAsync(C.d_vals.p, values, C.nnz * sizeof(double), cudaMemcpyHostToDevice, s));
    double anorm = 0;
    rc = dev_norm_frob(C, &anorm);
    if (rc) return rc;
    C.dparm[PGPU_DPARM_A_NORM] = anorm;
    // static pivoting threshold, sopalin/pastix_task_sopalin.c:461-485 (the
    // bcsc stays double, so eps = dlamch('e') also for the mixed factors)
    const double magn = C.dparm[PGPU_DPARM_EPSILON_MAGN_CTRL];
    double crit;
    if (magn < 0.) crit = -magn;
    else if (magn == 0.) crit = 1.1102230246251565e-16 * anorm;
    else crit = magn * anorm;
    k_gather_vals<<<1024, 256, 0, s>>>((int64_t)C.d_csr_val.n, C.d_csr_src.p, C.d_vals.p, C.d_csr_val.p);
    PGPU_CHECK(cudaMemsetAsync(C.d_status.p, 0, sizeof(Status), s));
    PGPU_CHECK(cudaMemsetAsync(C.d_coef.p, 0, ncoef * esz, s));
    int launches = 4;
    if (mixed)
        k_fillin<float><<<2048, 256, 0, s>>>(C.nnz, C.d_vals.p, C.d_fill_dst.p, (float *)C.d_coef.p, C.d_status.p);
    else
        k_fillin<double><<<2048, 256, 0, s>>>(C.nnz, C.d_vals.p, C.d_fill_dst.p, (double *)C.d_coef.p, C.d_status.p);
    int nl = 0;
    LaunchTimer tm(C);
    rc = mixed ? run_factor<float>(C, fact, crit, &nl, tm) : run_factor<double>(C, fact, crit, &nl, tm);
    if (rc) return rc;
    PGPU_CHECK(cudaEventRecord(C.ev[1], s));
    Status st;
    PGPU_CHECK(cudaMemcpyAsync(&st, C.d_status.p, sizeof(Status), cudaMemcpyDeviceToHost, s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[0], C.ev[1]));
    C.stats[0] = launches + nl;
    C.stats[3] = ms;
    {
        double ph[4];
        tm.collect(ph, 4);
        C.stats[8] = ph[PH_DIAG];
        C.stats[9] = ph[PH_TRSM];
        C.stats[6] = ph[PH_GEMM] + ph[PH_TC];
        C.stats[10] = C.gemm_flops[fact];
        C.stats[11] = ph[PH_TC];
        C.stats[12] = mixed ? C.tc_flops : 0.0;
        C.stats[13] = st.timeout;
    }
    if (st.timeout) {
        fprintf(stderr, "pastix_gpu: %d tensor-core GEMM tiles timed out waiting for their MMAs\n", st.timeout);
        C.fact_done = -1;
        return PASTIX_GPU_ERR_INTERNAL;
    }
    C.iparm[PGPU_IPARM_STATIC_PIVOTING] = st.nbpivots;
    const double fl = (fact == PGPU_FACT_GETRF) ? C.thflops_getrf : C.thflops_potrf;
    C.dparm[PGPU_DPARM_FACT_TIME] = ms * 1e-3;
    C.dparm[PGPU_DPARM_FACT_THFLOPS] = fl;
    C.dparm[PGPU_DPARM_FACT_FLOPS] = fl / (ms * 1e-3) / 1e9;
    C.coef_float = mixed;
    C.fact_done = fact;
    if (st.overflow) {
        fprintf(stderr, "pastix_gpu: mixed-precision overflow during the matrix initialization\n");
        C.fact_done = -1;
        return PASTIX_GPU_ERR_INTERNAL;
    }
    if (st.negpivots) fprintf(stderr, "pastix_gpu: Negative diagonal term (%d)\n", st.negpivots);
    if (st.nonfinite) {
        fprintf(stderr, "pastix_gpu: non-finite diagonal term met in the factorization (%d)\n", st.nonfinite);
        return PASTIX_GPU_ERR_INTERNAL;
    }
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// Solve on a permuted device RHS block W (factor precision, ld = n).
// --------------------------------------------------------------------------
template <typename T>
static int solve_permuted(pastix_gpu_t &C, T *W, int nrhs, int *launches) {
    const bool lu = (C.fact_done == PGPU_FACT_GETRF);
    const T *coefL = reinterpret_cast<const T *>(C.d_coef.p);
    const T *coefU = lu ? coefL + C.coefnbr : coefL;
    cudaStream_t s = C.stream;
    const int ldb = C.n;
    int nl = 0;
    PGPU_CHECK(cudaFuncSetAttribute(k_fwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(k_bwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(k_fwd_off<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    for (int l = 0; l < C.nlevels; l++) {
        const int ncb = C.lvl_ptr[l + 1] - C.lvl_ptr[l];
        const int mw = C.lvl_maxw[l];
        k_fwd_diag<T><<<ncb, 128, ((size_t)mw * nrhs + 32 * 33) * sizeof(T), s>>>(C.meta, C.d_lvl_cblks.p + C.lvl_ptr[l],
                                                                      coefL, W, ldb, nrhs, lu ? 1 : 0);
        nl++;
        const int nch = C.solve_ptr[l + 1] - C.solve_ptr[l];
        if (nch) {
            k_fwd_off<T><<<nch, 256, (size_t)mw * nrhs * sizeof(T), s>>>(
                C.meta, C.d_solve_chunks.p + C.solve_ptr[l], coefL, W, ldb, nrhs, SOLVE_ROWS_PER_CHUNK);
            nl++;
        }
    }
    for (int l = C.nlevels - 1; l >= 0; l--) {
        const int ncb = C.lvl_ptr[l + 1] - C.lvl_ptr[l];
        const int mw = C.lvl_maxw[l];
        const int nch = C.solve_ptr[l + 1] - C.solve_ptr[l];
        if (nch) {
            k_bwd_off<T><<<nch, 128, 0, s>>>(C.meta, C.d_solve_chunks.p + C.solve_ptr[l], coefU, W, ldb, nrhs,
                                              SOLVE_ROWS_PER_CHUNK);
            nl++;
        }
        k_bwd_diag<T><<<ncb, 128, ((size_t)mw * nrhs + 32 * 33) * sizeof(T), s>>>(C.meta, C.d_lvl_cblks.p + C.lvl_ptr[l],
                                                                      coefL, W, ldb, nrhs, lu ? 1 : 0);
        nl++;
    }
    PGPU_CHECK(cudaGetLastError());
    *launches += nl;
    return PASTIX_GPU_SUCCESS;
}

static int ensure_work(pastix_gpu_t &C) {
    const size_t need = (size_t)C.n * SOLVE_MAXRHS * sizeof(double);
    if (C.d_work.n < need) {
        C.d_work.release();
        PGPU_CHECK(C.d_work.alloc(need));
    }
    if (C.d_rhs.n < (size_t)C.n * SOLVE_MAXRHS) PGPU_CHECK(C.d_rhs.alloc((size_t)C.n * SOLVE_MAXRHS));
    return PASTIX_GPU_SUCCESS;
}

// Solve in place on a device FP64 block (user order, ld = ldb).
static int solve_device_block(pastix_gpu_t &C, double *dB, int64_t ldb, int nrhs, int *launches) {
    cudaStream_t s = C.stream;
    const int n = C.n;
    const int grid = std::min(4096, cdiv((int64_t)n * nrhs, 256));
    int rc;
    if (C.coef_float) {
        float *W = reinterpret_cast<float *>(C.d_work.p);
        k_permute<double, float><<<grid, 256, 0, s>>>(n, nrhs, C.d_peritab.p, dB, ldb, W, n, 0);
        rc = solve_permuted<float>(C, W, nrhs, launches);
        if (rc) return rc;
        k_permute<float, double><<<grid, 256, 0, s>>>(n, nrhs, C.d_peritab.p, W, n, dB, ldb, 1);
    } else {
        double *W = reinterpret_cast<double *>(C.d_work.p);
        k_permute<double, double><<<grid, 256, 0, s>>>(n, nrhs, C.d_peritab.p, dB, ldb, W, n, 0);
        rc = solve_permuted<double>(C, W, nrhs, launches);
        if (rc) return rc;
        k_permute<double, double><<<grid, 256, 0, s>>>(n, nrhs, C.d_peritab.p, W, n, dB, ldb, 1);
    }
    *launches += 2;
    PGPU_CHECK(cudaGetLastError());
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_solve(pastix_gpu_t *ctx, int64_t nrhs, void *B, int64_t ldb) {
    if (!ctx || !B || nrhs <= 0 || ldb < ctx->n) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (C.fact_done < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(C.device));
    int rc = ensure_work(C);
    if (rc) return rc;
    cudaStream_t s = C.stream;
    const bool dev = is_device_ptr(B);
    int launches = 0;
    PGPU_CHECK(cudaEventRecord(C.ev[2], s));
    for (int64_t r0 = 0; r0 < nrhs; r0 += SOLVE_MAXRHS) {
        const int nr = (int)std::min<int64_t>(SOLVE_MAXRHS, nrhs - r0);
        double *hb = reinterpret_cast<double *>(B) + r0 * ldb;
        double *db;
        int64_t dld;
        if (dev) {
            db = hb;
            dld = ldb;
        } else {
            db = C.d_rhs.p;
            dld = C.n;
            PGPU_CHECK(cudaMemcpy2DAsync(db, C.n * sizeof(double), hb, ldb * sizeof(double), C.n * sizeof(double),
                                         nr, cudaMemcpyHostToDevice, s));
        }
        rc = solve_device_block(C, db, dld, nr, &launches);
        if (rc) return rc;
        if (!dev)
            PGPU_CHECK(cudaMemcpy2DAsync(hb, ldb * sizeof(double), db, C.n * sizeof(double), C.n * sizeof(double),
                                         nr, cudaMemcpyDeviceToHost, s));
    }
    PGPU_CHECK(cudaEventRecord(C.ev[3], s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[2], C.ev[3]));
    C.stats[1] = launches;
    C.stats[4] = ms;
    C.dparm[PGPU_DPARM_SOLV_TIME] = ms * 1e-3;
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// Allocation-free solve (pastix_gpu_solve_noalloc): the permuted right-hand
// sides live in this file-scope device array instead of a cudaMalloc'ed
// workspace.  In host code `g_noalloc_scratch` only names the symbol; its
// device address comes from cudaGetSymbolAddress, looked up once per device
// (with that device current) on the first call there.
// --------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[PASTIX_GPU_NOALLOC_SCRATCH_BYTES];

namespace {
const int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {nullptr};
}  // namespace

// Device address of the scratch array on `dev` (the current device).
static int noalloc_scratch_address(int dev, void **addr) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return PASTIX_GPU_ERR_INTERNAL;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "pastix_gpu_solve_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return PASTIX_GPU_ERR_INTERNAL;
        }
        g_noalloc_addr[dev] = p;
    }
    *addr = g_noalloc_addr[dev];
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_solve_noalloc(pastix_gpu_t *ctx, int64_t nrhs, void *dB, int64_t ldb) {
    if (!ctx || !dB || nrhs <= 0 || ldb < ctx->n) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (C.fact_done < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    const size_t esz = C.coef_float ? sizeof(float) : sizeof(double);
    const size_t need = (size_t)C.n * (size_t)std::min<int64_t>(nrhs, SOLVE_MAXRHS) * esz;
    if (need > PASTIX_GPU_NOALLOC_SCRATCH_BYTES) {
        fprintf(stderr,
                "pastix_gpu_solve_noalloc: n=%d x %lld right-hand sides x %zu bytes = %zu bytes exceeds the "
                "%zu-byte scratch array\n",
                C.n, (long long)std::min<int64_t>(nrhs, SOLVE_MAXRHS), esz, need,
                (size_t)PASTIX_GPU_NOALLOC_SCRATCH_BYTES);
        return PASTIX_GPU_ERR_BADPARAMETER;
    }
    PGPU_CHECK(cudaSetDevice(C.device));
    if (!is_device_ptr(dB)) return PASTIX_GPU_ERR_BADPARAMETER;
    void *scratch = nullptr;
    int rc = noalloc_scratch_address(C.device, &scratch);
    if (rc) return rc;
    cudaStream_t s = C.stream;
    const int n = C.n;
    int launches = 0;
    for (int64_t r0 = 0; r0 < nrhs; r0 += SOLVE_MAXRHS) {
        const int nr = (int)std::min<int64_t>(SOLVE_MAXRHS, nrhs - r0);
        double *db = reinterpret_cast<double *>(dB) + r0 * ldb;
        const int grid = std::min(4096, cdiv((int64_t)n * nr, 256));
        if (C.coef_float) {
            float *W = reinterpret_cast<float *>(scratch);
            k_permute<double, float><<<grid, 256, 0, s>>>(n, nr, C.d_peritab.p, db, ldb, W, n, 0);
            rc = solve_permuted<float>(C, W, nr, &launches);
            if (rc) return rc;
            k_permute<float, double><<<grid, 256, 0, s>>>(n, nr, C.d_peritab.p, W, n, db, ldb, 1);
        } else {
            double *W = reinterpret_cast<double *>(scratch);
            k_permute<double, double><<<grid, 256, 0, s>>>(n, nr, C.d_peritab.p, db, ldb, W, n, 0);
            rc = solve_permuted<double>(C, W, nr, &launches);
            if (rc) return rc;
            k_permute<double, double><<<grid, 256, 0, s>>>(n, nr, C.d_peritab.p, W, n, db, ldb, 1);
        }
    }
    PGPU_CHECK(cudaGetLastError());
    PGPU_CHECK(cudaStreamSynchronize(s));
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// Refinement (refinement/z_refine_grad.c:49 z_grad_smp, preconditioned CG).
// Vectors in the user numbering (the SpMV matrix is permuted, so vectors are
// permuted in and out of it).
// --------------------------------------------------------------------------
struct VecOps {
    pastix_gpu_t &C;
    int launches = 0;
    double dot(const double *x, const double *y) {
        const int nb = 256;
        k_dot_partial<<<nb, RED_THREADS, 0, C.stream>>>(C.n, x, y, C.d_partial.p);
        k_dot_final<<<1, RED_THREADS, 0, C.stream>>>(nb, C.d_partial.p, C.d_scalar.p, 0);
        launches += 2;
        double v = 0;
        cudaMemcpyAsync(&v, C.d_scalar.p, sizeof(double), cudaMemcpyDeviceToHost, C.stream);
        cudaStreamSynchronize(C.stream);
        return v;
    }
    double norm(const double *x) { return std::sqrt(dot(x, nullptr)); }
    void axpy(double a, const double *x, double *y) {
        k_axpy<<<1024, 256, 0, C.stream>>>(C.n, a, x, y);
        launches++;
    }
    void xpby(const double *z, double beta, double *p) {
        k_xpby<<<1024, 256, 0, C.stream>>>(C.n, z, beta, p);
        launches++;
    }
    void copy(const double *x, double *y) {
        cudaMemcpyAsync(y, x, C.n * sizeof(double), cudaMemcpyDeviceToDevice, C.stream);
    }
    // y = alpha A x + beta y, in the user numbering: the CSR is permuted, so
    // work on permuted copies held in d_gm.
    void spmv(double alpha, const double *x, double beta, double *y) {
        const int n = C.n;
        double *xp = C.d_gm.p, *yp = C.d_gm.p + n;
        const int grid = cdiv(n, 256);
        k_permute<double, double><<<grid, 256, 0, C.stream>>>(n, 1, C.d_peritab.p, x, n, xp, n, 0);
        if (beta != 0.0) k_permute<double, double><<<grid, 256, 0, C.stream>>>(n, 1, C.d_peritab.p, y, n, yp, n, 0);
        k_spmv<<<cdiv((int64_t)n * 32, 256), 256, 0, C.stream>>>(n, C.d_csr_ptr.p, C.d_csr_col.p, C.d_csr_val.p,
                                                                alpha, xp, beta, yp);
        k_permute<double, double><<<grid, 256, 0, C.stream>>>(n, 1, C.d_peritab.p, yp, n, y, n, 1);
        launches += 3 + (beta != 0.0);
    }
    int spsv(double *z) { return solve_device_block(C, z, C.n, 1, &launches); }
};

static int refine_cg(pastix_gpu_t &C, VecOps &V, const double *b, double *x, double eps, int itermax, int *iters,
                     double *resid) {
    const int n = C.n;
    double *r = C.d_r.p, *z = C.d_z.p, *p = C.d_p.p, *ap = C.d_ap.p;
    double normb = V.norm(b);
    if (normb == 0.) normb = 1;
    const double normx = V.norm(x);
    V.copy(b, r);
    if (normx > 0.) V.spmv(-1.0, x, 1.0, r);
    double normr = V.norm(r);
    double resid_b = normr / normb;
    V.copy(r, z);
    int rc = V.spsv(z);
    if (rc) return rc;
    V.copy(z, p);
    int it = 0;
    (void)n;
    while (resid_b > eps && it < itermax) {
        it++;
        V.spmv(1.0, p, 0.0, ap);
        double beta = V.dot(r, z);
        double alpha = V.dot(ap, p);
        alpha = beta / alpha;
        V.axpy(alpha, p, x);
        V.axpy(-alpha, ap, r);
        V.copy(r, z);
        rc = V.spsv(z);
        if (rc) return rc;
        alpha = V.dot(r, z);
        beta = alpha / beta;
        V.xpby(z, beta, p);
        normr = V.norm(r);
        resid_b = normr / normb;
    }
    *iters = it;
    *resid = resid_b;
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// GMRES(im), right preconditioned (refinement/z_refine_gmres.c:49
// z_gmres_smp, Saad Alg. 9.5): V holds the Krylov basis, W = M^{-1} V so the
// solution update needs no extra solve; modified Gram-Schmidt with the
// projections h_{j,i} kept in device memory (one host round trip per inner
// iteration, for the Givens rotations on the small Hessenberg matrix).
// --------------------------------------------------------------------------
static int refine_gmres(pastix_gpu_t &C, VecOps &V, const double *b, double *x, double eps, int itermax, int im,
                        int *iters_out, double *resid_out) {
    const int64_t n = C.n;
    const int im1 = im + 1;
    if (C.d_gmV.n < (size_t)n * im1) {
        PGPU_CHECK(C.d_gmV.alloc((size_t)n * im1));
        PGPU_CHECK(C.d_gmW.alloc((size_t)n * im));
    }
    if (C.d_gmh.n < (size_t)2 * im1) PGPU_CHECK(C.d_gmh.alloc((size_t)2 * im1));
    cudaStream_t s = C.stream;
    double *gV = C.d_gmV.p, *gW = C.d_gmW.p, *dh = C.d_gmh.p;
    std::vector<double> H((size_t)im * im1, 0.0), cs(im, 0.0), sn(im, 0.0), G(im1, 0.0), hcol(im1, 0.0);
    double normb = V.norm(b);
    if (normb == 0.) normb = 1;
    const double normx = V.norm(x);
    int iters = 0;
    double resid_b = 0;
    bool outflag = true;
    while (outflag) {
        // r0 = b - A x
        V.copy(b, gV);
        if (normx > 0. || iters > 0) V.spmv(-1.0, x, 1.0, gV);
        double resid = V.norm(gV);
        resid_b = resid / normb;
        if (resid_b <= eps) break;
        k_scal<<<1024, 256, 0, s>>>(n, 1.0 / resid, gV);
        V.launches++;
        std::fill(G.begin(), G.end(), 0.0);
        G[0] = resid;
        int i = -1;
        bool inflag = true;
        while (inflag) {
            i++;
            double *vi = gV + (int64_t)i * n, *wi = gW + (int64_t)i * n, *vn = gV + (int64_t)(i + 1) * n;
            V.copy(vi, wi);
            int rc = V.spsv(wi);                       // w_i = M^{-1} v_i
            if (rc) return rc;
            V.spmv(1.0, wi, 0.0, vn);                  // v_{i+1} = A w_i
            for (int j = 0; j <= i; j++) {             // modified Gram-Schmidt
                k_dot_partial<<<256, RED_THREADS, 0, s>>>(n, vn, gV + (int64_t)j * n, C.d_partial.p);
                k_dot_final<<<1, RED_THREADS, 0, s>>>(256, C.d_partial.p, dh + j, 0);
                k_axpy_dev<<<1024, 256, 0, s>>>(n, dh + j, -1.0, gV + (int64_t)j * n, vn);
                V.launches += 3;
            }
            k_dot_partial<<<256, RED_THREADS, 0, s>>>(n, vn, nullptr, C.d_partial.p);
            k_dot_final<<<1, RED_THREADS, 0, s>>>(256, C.d_partial.p, dh + i + 1, 1);
            V.launches += 2;
            PGPU_CHECK(cudaMemcpyAsync(hcol.data(), dh, (i + 2) * sizeof(double), cudaMemcpyDeviceToHost, s));
            PGPU_CHECK(cudaStreamSynchronize(s));
            const double norm = hcol[i + 1];
            if (norm > 1e-50) {
                k_scal<<<1024, 256, 0, s>>>(n, 1.0 / norm, vn);
                V.launches++;
            }
            double *Hi = H.data() + (size_t)i * im1;
            for (int j = 0; j <= i + 1; j++) Hi[j] = hcol[j];
            for (int j = 0; j < i; j++) {              // previous Givens rotations
                const double tmp = Hi[j];
                Hi[j] = cs[j] * tmp + sn[j] * Hi[j + 1];
                Hi[j + 1] = cs[j] * Hi[j + 1] - sn[j] * tmp;
            }
            double t = std::sqrt(Hi[i] * Hi[i] + Hi[i + 1] * Hi[i + 1]);
            if (std::fabs(t) <= eps) t = eps;
            cs[i] = Hi[i] / t;
            sn[i] = Hi[i + 1] / t;
            G[i + 1] = -sn[i] * G[i];
            G[i] = cs[i] * G[i];
            Hi[i] = cs[i] * Hi[i] + sn[i] * Hi[i + 1];
            resid = std::fabs(G[i + 1]);
            resid_b = resid / normb;
            iters++;
            if (i + 1 >= im || resid_b <= eps || iters >= itermax) inflag = false;
        }
        // y = H^{-1} g (upper triangular, size i+1), x += W y
        const int k = i + 1;
        for (int r = k - 1; r >= 0; r--) {
            double sum = G[r];
            for (int j = r + 1; j < k; j++) sum -= H[(size_t)j * im1 + r] * G[j];
            G[r] = sum / H[(size_t)r * im1 + r];
        }
        PGPU_CHECK(cudaMemcpyAsync(dh, G.data(), k * sizeof(double), cudaMemcpyHostToDevice, s));
        k_gemv_acc<<<1024, 256, 0, s>>>(n, k, gW, n, dh, x);
        V.launches++;
        PGPU_CHECK(cudaStreamSynchronize(s));
        if (iters >= itermax) outflag = false;
    }
    *iters_out = iters;
    *resid_out = resid_b;
    return PASTIX_GPU_SUCCESS;
}

static int ensure_refine_vectors(pastix_gpu_t &C) {
    const size_t n = C.n;
    if (C.d_r.n < n) {
        PGPU_CHECK(C.d_r.alloc(n));
        PGPU_CHECK(C.d_z.alloc(n));
        PGPU_CHECK(C.d_p.alloc(n));
        PGPU_CHECK(C.d_ap.alloc(n));
        PGPU_CHECK(C.d_x.alloc(n));
        PGPU_CHECK(C.d_gm.alloc(2 * n));
    }
    return ensure_work(C);
}

static int refine_impl(pastix_gpu_t &C, int64_t nrhs, const void *B, int64_t ldb, void *X, int64_t ldx) {
    int rc = ensure_refine_vectors(C);
    if (rc) return rc;
    cudaStream_t s = C.stream;
    double eps = C.dparm[PGPU_DPARM_EPSILON_REFINEMENT];
    if (eps < 0.) eps = 1e-12;   // refinement/pastix_task_refine.c:131-140 (double input)
    const int itermax = (int)C.iparm[PGPU_IPARM_ITERMAX];
    const int method = (int)C.iparm[PGPU_IPARM_REFINEMENT];
    if (method != PGPU_REFINE_CG && method != PGPU_REFINE_GMRES) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    const int im = std::max<int>(1, (int)C.iparm[PGPU_IPARM_GMRES_IM]);
    const bool bdev = is_device_ptr(B), xdev = is_device_ptr(X);
    VecOps V{C};
    int maxit = 0;
    double maxres = 0;
    PGPU_CHECK(cudaEventRecord(C.ev[4], s));
    for (int64_t r = 0; r < nrhs; r++) {
        const double *bcol = reinterpret_cast<const double *>(B) + r * ldb;
        double *xcol = reinterpret_cast<double *>(X) + r * ldx;
        double *db = C.d_rhs.p, *dx = C.d_x.p;
        PGPU_CHECK(cudaMemcpyAsync(db, bcol, C.n * sizeof(double),
                                   bdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        PGPU_CHECK(cudaMemcpyAsync(dx, xcol, C.n * sizeof(double),
                                   xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        int it = 0;
        double res = 0;
        rc = (method == PGPU_REFINE_CG) ? refine_cg(C, V, db, dx, eps, itermax, &it, &res)
                                        : refine_gmres(C, V, db, dx, eps, itermax, im, &it, &res);
        if (rc) return rc;
        PGPU_CHECK(cudaMemcpyAsync(xcol, dx, C.n * sizeof(double),
                                   xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
        maxit = std::max(maxit, it);
        maxres = std::max(maxres, res);
    }
    PGPU_CHECK(cudaEventRecord(C.ev[5], s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[4], C.ev[5]));
    C.stats[2] = V.launches;
    C.stats[5] = ms;
    C.iparm[PGPU_IPARM_NBITER] = maxit;
    C.dparm[PGPU_DPARM_RELATIVE_ERROR] = maxres;
    C.dparm[PGPU_DPARM_REFINE_TIME] = ms * 1e-3;
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_refine(pastix_gpu_t *ctx, int64_t nrhs, const void *B, int64_t ldb, void *X,
                                 int64_t ldx) {
    if (!ctx || !B || !X || nrhs <= 0 || ldb < ctx->n || ldx < ctx->n) return PASTIX_GPU_ERR_BADPARAMETER;
    if (ctx->fact_done < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(ctx->device));
    return refine_impl(*ctx, nrhs, B, ldb, X, ldx);
}

extern "C" int pastix_gpu_solve_and_refine(pastix_gpu_t *ctx, int64_t nrhs, const void *B, int64_t ldb, void *X,
                                           int64_t ldx) {
    if (!ctx || !B || !X || nrhs <= 0 || ldb < ctx->n || ldx < ctx->n) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (C.fact_done < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(C.device));
    const bool bdev = is_device_ptr(B), xdev = is_device_ptr(X);
    if (bdev && xdev) {
        // X := B, solve in place, then refine -- all on the device
        PGPU_CHECK(cudaMemcpy2DAsync(X, ldx * sizeof(double), B, ldb * sizeof(double), C.n * sizeof(double), nrhs,
                                     cudaMemcpyDeviceToDevice, C.stream));
        int rc = pastix_gpu_solve(ctx, nrhs, X, ldx);
        if (rc) return rc;
        return refine_impl(C, nrhs, B, ldb, X, ldx);
    }
    // host buffers: B crosses once, X comes back once
    if (C.d_sr_b.n < (size_t)C.n * nrhs) {
        PGPU_CHECK(C.d_sr_b.alloc((size_t)C.n * nrhs));
        PGPU_CHECK(C.d_sr_x.alloc((size_t)C.n * nrhs));
    }
    double *db = C.d_sr_b.p, *dx = C.d_sr_x.p;
    PGPU_CHECK(cudaMemcpy2DAsync(db, C.n * sizeof(double), B, ldb * sizeof(double), C.n * sizeof(double), nrhs,
                                 bdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, C.stream));
    PGPU_CHECK(cudaMemcpyAsync(dx, db, (size_t)C.n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, C.stream));
    int rc = pastix_gpu_solve(ctx, nrhs, dx, C.n);
    if (rc) return rc;
    rc = refine_impl(C, nrhs, db, C.n, dx, C.n);
    if (rc) return rc;
    PGPU_CHECK(cudaMemcpy2DAsync(X, ldx * sizeof(double), dx, C.n * sizeof(double), C.n * sizeof(double), nrhs,
                                 xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, C.stream));
    PGPU_CHECK(cudaStreamSynchronize(C.stream));
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_get_params(pastix_gpu_t *ctx, int64_t *iparm, double *dparm) {
    if (!ctx) return PASTIX_GPU_ERR_BADPARAMETER;
    if (iparm) std::memcpy(iparm, ctx->iparm, sizeof(ctx->iparm));
    if (dparm) std::memcpy(dparm, ctx->dparm, sizeof(ctx->dparm));
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_set_iparm(pastix_gpu_t *ctx, int index, int64_t value) {
    if (!ctx || index < 0 || index >= PGPU_IPARM_SIZE) return PASTIX_GPU_ERR_BADPARAMETER;
    ctx->iparm[index] = value;
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_set_dparm(pastix_gpu_t *ctx, int index, double value) {
    if (!ctx || index < 0 || index >= PGPU_DPARM_SIZE) return PASTIX_GPU_ERR_BADPARAMETER;
    ctx->dparm[index] = value;
    return PASTIX_GPU_SUCCESS;
}

// Factors in the reference's 1D layout (column-major stride x width panels).
template <typename T>
static void host_relayout(const pastix_gpu_t &C, const std::vector<T> &dev, T *L, T *U, bool lu) {
    int64_t off = 0;
    for (int c = 0; c < C.cblknbr; c++) {
        const int w = C.width[c], h = C.height[c], ld = C.ld[c];
        const T *P = dev.data() + C.coefoff[c];
        const T *PU = dev.data() + C.coefnbr + C.coefoff[c];
        for (int j = 0; j < w; j++)
            for (int i = 0; i < h; i++) {
                if (L) L[off + (int64_t)j * h + i] = P[(int64_t)i * ld + j];
                if (lu && U) U[off + (int64_t)j * h + i] = (i < w) ? P[(int64_t)j * ld + i] : PU[(int64_t)i * ld + j];
            }
        off += (int64_t)h * w;
    }
}

extern "C" int pastix_gpu_coeftab(pastix_gpu_t *ctx, void *L, void *U) {
    if (!ctx || ctx->fact_done < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    PGPU_CHECK(cudaSetDevice(C.device));
    const bool lu = (C.fact_done == PGPU_FACT_GETRF);
    const size_t ncoef = (size_t)C.coefnbr * (lu ? 2 : 1);
    if (C.coef_float) {
        std::vector<float> h(ncoef);
        PGPU_CHECK(cudaMemcpy(h.data(), C.d_coef.p, ncoef * sizeof(float), cudaMemcpyDeviceToHost));
        host_relayout<float>(C, h, (float *)L, (float *)U, lu);
    } else {
        std::vector<double> h(ncoef);
        PGPU_CHECK(cudaMemcpy(h.data(), C.d_coef.p, ncoef * sizeof(double), cudaMemcpyDeviceToHost));
        host_relayout<double>(C, h, (double *)L, (double *)U, lu);
    }
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_stats(pastix_gpu_t *ctx, double *stats) {
    if (!ctx || !stats) return PASTIX_GPU_ERR_BADPARAMETER;
    std::memcpy(stats, ctx->stats, sizeof(ctx->stats));
    return PASTIX_GPU_SUCCESS;
}

extern "C" void pastix_gpu_finalize(pastix_gpu_t **pctx) {
    if (!pctx || !*pctx) return;
    pastix_gpu_t *C = *pctx;
    cudaSetDevice(C->device);
    if (C->stream) cudaStreamSynchronize(C->stream);
    for (auto &e : C->ev) cudaEventDestroy(e);
    for (auto &e : C->evpool) cudaEventDestroy(e);
    if (C->stream) cudaStreamDestroy(C->stream);
    delete C;   // every DArr member frees its device memory
    *pctx = nullptr;
}
