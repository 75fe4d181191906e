// Host side of the B200 sopalin replacement: the C ABI declared in
// include/pastix_gpu.h, the device layout of the coeftab, the level schedule
// and the drivers of numfact / solve / refinement.
#include "pastix_gpu.h"
#include "pgpu_factor.cuh"
#include "pgpu_solve.cuh"
#include "pgpu_panel.cuh"
#include "pgpu_gemm_tc.cuh"
#include "pgpu_panel_wide.cuh"
#include "pgpu_gemm_tma.cuh"
#include "pgpu_gemm_f64.cuh"
#include "pgpu_spm.cuh"
#include "pgpu_solve_flow.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <cudaTypedefs.h>

#include <algorithm>
#include <queue>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <unordered_map>
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
const int SOLVE_SMALL_MAXH = 512;   // tallest cblk of a level solved one warp per cblk

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
    std::vector<int> lvl_ptr, lvl_cblks, lvl_maxw, lvl_maxh, cblk_level;
    // lookahead: the update tiles of a level that target the next level run
    // on the main stream, the others on stream2, overlapping the panels of
    // the levels that follow
    cudaStream_t stream2 = nullptr;
    std::vector<cudaEvent_t> la_events;
    std::vector<int> tile_crit, tctile_crit;   // per level: critical (next-level) tiles first
    double side_ms[4] = {0};                   // stream2 GEMM time of the last numfact, per phase
    // CUDA graph of the factorization sequence (norm .. last level), replayed
    // while the plan, the coeftab and the value buffers stay the same
    bool capturing = false;
    cudaGraph_t fact_graph = nullptr;
    cudaGraphExec_t fact_exec = nullptr;
    std::vector<int> g_kinds, g_kinds2;   // the captured graph's timing marks (evpool, evpool2)
    int g_used = 0, g_used2 = 0, g_nl = 0;
    int64_t graph_key[5] = {-1, -1, -1, -1, -1};
    double thflops[2][3] = {{0}};   // [complex][POTRF, GETRF, LDL] algorithmic flops

    // ---- device structure ----
    DArr<int> d_fcol, d_width, d_height, d_ld, d_fblok, d_rowidx, d_bfrow, d_blrow, d_browoff, d_bfcblk,
        d_lvl_cblks, d_peritab;
    DArr<int64_t> d_coefoff, d_rowbase;
    Meta meta{};

    // ---- factorization plan (per factotype) ----
    int plan_fact = -1;
    std::vector<int> tile_ptr, tctile_ptr, trsm_ptr, lvl_plrows, lvl_porows;
    std::vector<int> stile_n;   // per level and part (next-level targets, others): warp tiles at the part's end
    // panel launches of a level: k_panel_factor over the narrow cblks and
    // k_panel_wide over the wide diagonal blocks, jobs {cblk, position in
    // lvl_cblks} (the position indexes the task records)
    std::vector<int> pn_ptr, pw_ptr, lvl_pmaxw, lvl_wmaxw;
    DArr<int2> d_pjobs, d_wjobs;
    std::vector<int> ps_ptr;   // cblks of at most 32 columns: one warp each (k_panel_small)
    DArr<int2> d_sjobs;
    DArr<int4> d_tiles, d_tctiles, d_trsm;
    double tc_flops = 0;   // update-GEMM flops on the tensor-core path
    DArr<GemmTask> d_tasks;
    std::vector<int> solve_ptr;
    DArr<int2> d_solve_chunks;

    // ---- matrix ----
    int mtxtype = PGPU_SYMMETRIC, flttype = PGPU_DOUBLE;
    int64_t nnz = 0, csr_nnz = 0;
    DArr<int64_t> d_fill_dst;   // per user nnz: coeftab offset (U entries offset by coefnbr), ~offset: conjugate
    DArr<int8_t> d_wgt;         // Frobenius weight per user nnz
    DArr<int64_t> d_csr_ptr, d_csr_src;
    DArr<int> d_csr_col;
    DArr<double> d_csr_val, d_vals;
    bool have_spm = false;

    // ---- tuning (pastix_gpu_set_tuning; the autotuner's knobs) ----
    int64_t tune[PGPU_TUNE_COUNT] = {0};

    // ---- numerical state ----
    DArr<unsigned char> d_coef;
    int coef_float = 0;     // factor precision of d_coef
    int fact_done = -1;     // factotype of the factors in d_coef, -1 if none
    int fact_mode = -1;     // kernel form (FM_*) of those factors
    DArr<Status> d_status;
    DArr<double> d_partial, d_scalar;
    DArr<unsigned char> d_work;   // solve workspace (n x 16 in factor precision)
    DArr<double> d_rhs, d_x, d_r, d_z, d_p, d_ap, d_gm;   // refinement vectors
    DArr<double> d_sr_b, d_sr_x;   // solve_and_refine staging of host B / X
    DArr<double> d_gmV, d_gmW, d_gmh;   // GMRES basis, preconditioned basis, projections
    std::vector<int64_t> seg;           // batch: first unknown of each system (+ n), empty if none
    DArr<int64_t> d_seg;
    DArr<double> d_segss;               // per-system sums of squares
    std::vector<cudaEvent_t> evpool, evpool2;   // per-launch timing events (solves; the numfact's stream2)
    std::vector<cudaEvent_t> evpoolf;           // the numfact's main-stream timing events
    // phase timeline of the last directly launched numfact (pastix_gpu_phase_log):
    // {stream, phase, level} and {start, end} ms from the numfact's first event
    std::vector<int> log_kinds, log_levels, log_kinds2, log_levels2;
    int log_used = 0, log_used2 = 0;
    // the numfact's per-phase times and timeline are read from its events when
    // first asked for (pastix_gpu_stats / pastix_gpu_phase_log), not between the
    // numfact and the next call: 1 direct launch, 2 graph replay, 0 collected
    int fact_marks_pending = 0;
    std::vector<int64_t> phase_info;
    std::vector<double> phase_times;
    DArr<double> d_fact_scal;          // [0] ||A||_F, [1] static-pivot threshold (device-side, no host trip)
    // per-task timings of the last numfact (learned cost model), when record
    bool record = false;
    DArr<int64_t> d_prof[4];           // panel CTAs, TRSM chunks, FMA GEMM tiles, tensor-core tiles
    // panel TRSM as a GEMM against the inverse of the diagonal block (big panels of LL^t / LDL)
    bool trsm_gemm = false;
    std::vector<int64_t> invoff, scroff;
    DArr<int64_t> d_invoff, d_scroff;
    DArr<unsigned char> d_inv, d_scr;    // inverse workspace (zeroed), per-level TRSM output
    // TMA operands of the tensor-core GEMMs: hi/lo mirrors [2][plane] of the
    // coeftab and of the inverses (3xTF32), one tensor map per (source cblk,
    // operand kind), split jobs {cblk, row, panel, -} per level
    bool tma = false;
    DArr<float> d_hilo, d_ihilo;
    // 3xFP16 operands (mixed GEMM mode 3): FP16 hi / lo planes [2][h16_plane]
    // of the source matrices, per-row inverse scales, and per operand map its
    // first element (d_hoff) and first scale (d_hsbase)
    bool h16 = false;
    DArr<__half> d_h16;
    DArr<float> d_hscale;
    DArr<int64_t> d_hoff, d_hsbase;
    int64_t h16_plane = 0;
    // per task {target-row map base, A row-scale base, B row-scale base} and
    // the target rows of the tensor-core update tasks (k_task_rowmap)
    DArr<int64_t> d_taux;
    DArr<int> d_tmap, d_tlist;
    DArr<TcDesc> d_tcdesc, d_ttdesc;   // per tensor-core tile (update, TRSM): k_gemm_scatter_tc_tma's records
    // dataflow solve of runs of levels whose cblks all hold a diagonal-block
    // inverse (k_solve_flow): runs {first level, end level}, per run the task
    // ranges (forward, backward), the per-cblk counters (5 x cblknbr) and their
    // per-launch increments (4 x cblknbr), epochs and ticket bases, the Y and Z
    // blocks (n x FLOW_MAXRHS each), the largest width of a run's cblk
    std::vector<int2> flow_runs;
    std::vector<int> flow_tptr[2];    // per run: first task
    DArr<int> d_flow_off[2];          // per run: 2 x (G + 1) offsets of the CTAs' tasks in the two lists
    int flow_G = 0;
    DArr<FlowTask> d_flow_tasks[2];
    DArr<unsigned long long> d_flow_cnt;
    DArr<int> d_flow_need;
    DArr<FlowState> d_flow_state;
    DArr<unsigned char> d_flowY, d_flowZ;
    DArr<unsigned long long> d_flow_stamps;   // per-task times of the last launch (PASTIX_GPU_SOLVE_PROFILE=3)
    std::vector<unsigned long long> flow_epoch[2];
    int flow_maxw = 0;
    bool flow_used = false;
    int64_t hilo_plane = 0, ihilo_plane = 0;
    DArr<CUtensorMap> d_tmaps;
    DArr<int> d_mapidx;
    std::vector<int> split_ptr;
    DArr<int4> d_split;
    std::vector<int> inv_ptr, ttile_ptr, tttile_ptr;   // per level: inverse jobs, TRSM FMA / TC tiles
    DArr<int2> d_invjobs;
    DArr<int4> d_ttiles, d_tttiles;
    std::vector<int4> h_tiles, h_tctiles, h_trsm;   // host copies of the plan's launch lists
    std::vector<GemmTask> h_tasks;
    int plan_fuse = 0, plan_esz = 0, plan_fmode = -1;
    double plan_gemm_flops = 0;        // update-GEMM flops of the current plan
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

static void default_tuning(int64_t *t);

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
    default_tuning(ctx->tune);
    if (iparm) std::memcpy(ctx->iparm, iparm, sizeof(ctx->iparm));
    if (dparm) std::memcpy(ctx->dparm, dparm, sizeof(ctx->dparm));
    int prio_lo = 0, prio_hi = 0;
    PGPU_CHECK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    PGPU_CHECK(cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_hi));
    PGPU_CHECK(cudaStreamCreateWithPriority(&ctx->stream2, cudaStreamNonBlocking, prio_lo));
    for (auto &e : ctx->ev) PGPU_CHECK(cudaEventCreate(&e));
    PGPU_CHECK(ctx->d_status.alloc(1));
    PGPU_CHECK(ctx->d_partial.alloc(1024));
    PGPU_CHECK(ctx->d_scalar.alloc(16));
    PGPU_CHECK(ctx->d_fact_scal.alloc(4));
    PGPU_CHECK(ctx->d_flow_state.alloc(1));
    PGPU_CHECK(cudaMemset(ctx->d_flow_state.p, 0, sizeof(FlowState)));
    *pctx = ctx;
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// Algorithmic flops of the factorization (DPARM_FACT_THFLOPS), the
// reference's model: symbol/symbol_cost.c:422 pastixSymbolGetFlops sums
// sum1d per cblk -- diag(N) + trsm(M, N) + update(N, M) with N = width,
// M = off-diagonal rows -- over symbol/symbol_cost_flops.c flopstable, with
// the operation counts of common/flops.h (complex: 6 flops per multiply, 2
// per add).  form: 0 POTRF, 1 GETRF, 2 LDL.
// --------------------------------------------------------------------------
static double structure_flops(const pastix_gpu_t &C, int form, bool z) {
    auto fl = [z](double mul, double add) { return z ? 6.0 * mul + 2.0 * add : mul + add; };
    const double scalw = z ? 6.0 : 1.0;
    double tot = 0;
    for (int c = 0; c < C.cblknbr; c++) {
        const double N = C.width[c], M = C.height[c] - C.width[c];
        if (form == 0) tot += fl(N * ((N / 6.0 + 0.5) * N + 1.0 / 3.0), N * ((N / 6.0) * N - 1.0 / 6.0));
        else if (form == 1) tot += fl(0.5 * N * (N * (N - N / 3.0 - 1.0) + N) + 2.0 / 3.0 * N,
                                     0.5 * N * (N * (N - N / 3.0) - N) + N / 6.0);
        else tot += fl(N * ((N / 6.0 + 0.5) * N + 10.0 / 3.0), N * ((N / 6.0) * N - 1.0 / 6.0));
        if (M <= 0) continue;
        const double trsm = fl(0.5 * M * N * (N + 1), 0.5 * M * N * (N + 1));   // FLOPS_TRSM(Right, M, N)
        const double syrk = fl(0.5 * N * M * (M + 1), 0.5 * N * M * (M + 1));   // FLOPS_SYRK(N, M)
        if (form == 0) tot += trsm + syrk;
        else if (form == 1) tot += 2.0 * trsm + fl(M * M * N, M * M * N);     // + FLOPS_GEMM(M, M, N)
        else tot += trsm + scalw * N * M + syrk + scalw * M * M;
    }
    return tot;
}

// --------------------------------------------------------------------------
// Structure handoff: device layout + level schedule.
// --------------------------------------------------------------------------
static void invalidate_graph(pastix_gpu_t &C);

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
    for (int z = 0; z < 2; z++)
        for (int f = 0; f < 3; f++) C.thflops[z][f] = structure_flops(C, f, z != 0);
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
    C.cblk_level = level;
    C.lvl_ptr.assign(C.nlevels + 1, 0);
    for (int c = 0; c < nc; c++) C.lvl_ptr[level[c] + 1]++;
    for (int l = 0; l < C.nlevels; l++) C.lvl_ptr[l + 1] += C.lvl_ptr[l];
    C.lvl_cblks.assign(nc, 0);
    C.lvl_maxw.assign(C.nlevels, 0);
    C.lvl_maxh.assign(C.nlevels, 0);
    {
        std::vector<int> pos(C.lvl_ptr.begin(), C.lvl_ptr.end() - 1);
        for (int c = 0; c < nc; c++) {
            C.lvl_cblks[pos[level[c]]++] = c;
            C.lvl_maxw[level[c]] = std::max(C.lvl_maxw[level[c]], C.width[c]);
            C.lvl_maxh[level[c]] = std::max(C.lvl_maxh[level[c]], C.height[c]);
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
    C.invoff.assign(nc, -1);
    PGPU_CHECK(C.d_invoff.upload(C.invoff, s));
    C.meta = Meta{C.n, nc, nb, C.d_fcol.p, C.d_width.p, C.d_height.p, C.d_ld.p, C.d_coefoff.p,
                  C.d_fblok.p, C.d_rowbase.p, C.d_rowidx.p, C.d_bfrow.p, C.d_blrow.p, C.d_browoff.p,
                  C.d_bfcblk.p, C.d_invoff.p};

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


// --------------------------------------------------------------------------
// Pattern handoff: fill-in map (bcsc -> coeftab) and the permuted CSR.
// --------------------------------------------------------------------------
extern "C" int pastix_gpu_spm(pastix_gpu_t *ctx, int mtxtype, int flttype, int64_t n, const int64_t *colptr,
                              const int64_t *rowptr) {
    if (!ctx || !colptr || !rowptr) return PASTIX_GPU_ERR_BADPARAMETER;
    if (n != ctx->n) return PASTIX_GPU_ERR_BADPARAMETER;
    if (flttype != PGPU_DOUBLE && flttype != PGPU_COMPLEX64) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    if (mtxtype != PGPU_GENERAL && mtxtype != PGPU_SYMMETRIC && mtxtype != PGPU_HERMITIAN)
        return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(ctx->device));
    auto &C = *ctx;
    invalidate_graph(C);   // the value maps below are reallocated
    C.mtxtype = mtxtype;
    C.flttype = flttype;
    const int64_t nnz = colptr[n];
    if (nnz < 0 || 2 * nnz > (int64_t)INT32_MAX) return PASTIX_GPU_ERR_BADPARAMETER;
    C.nnz = nnz;
    const bool sym = (mtxtype != PGPU_GENERAL);
    // a Hermitian entry that lands in the other triangle is stored conjugated
    const bool herm = (mtxtype == PGPU_HERMITIAN && flttype == PGPU_COMPLEX64);
    cudaStream_t s = C.stream;
    PGPU_CHECK(cudaEventRecord(C.ev[4], s));
    // the pattern, the ordering and the column -> cblk map go to the device;
    // the maps are built there (k_spm_maps, a stable radix sort by row, k_spm_csr)
    std::vector<int> perm(n);
    for (int k = 0; k < n; k++) perm[C.peritab[k]] = k;
    DArr<int64_t> d_colptr, d_rowptr, d_slot, d_sslot;
    DArr<int> d_perm, d_c2c, d_key, d_skey, d_colof, d_bad;
    DArr<unsigned char> d_tmp;
    {
        std::vector<int64_t> cp(colptr, colptr + n + 1), rp(rowptr, rowptr + nnz);
        PGPU_CHECK(d_colptr.upload(cp, s));
        PGPU_CHECK(d_rowptr.upload(rp, s));
        PGPU_CHECK(d_perm.upload(perm, s));
        PGPU_CHECK(d_c2c.upload(C.col2cblk, s));
        PGPU_CHECK(cudaStreamSynchronize(s));   // (the host vectors leave scope)
    }
    const int64_t ns = 2 * std::max<int64_t>(nnz, 1);
    PGPU_CHECK(C.d_fill_dst.alloc(std::max<int64_t>(nnz, 1)));
    PGPU_CHECK(C.d_wgt.alloc(std::max<int64_t>(nnz, 1)));
    PGPU_CHECK(d_key.alloc(ns));
    PGPU_CHECK(d_skey.alloc(ns));
    PGPU_CHECK(d_slot.alloc(ns));
    PGPU_CHECK(d_sslot.alloc(ns));
    PGPU_CHECK(d_colof.alloc(std::max<int64_t>(nnz, 1)));
    PGPU_CHECK(d_bad.alloc(1));
    PGPU_CHECK(cudaMemsetAsync(d_bad.p, 0, sizeof(int), s));
    SpmMaps sm{(int)n, nnz, sym ? 1 : 0, herm ? 1 : 0, d_colptr.p, d_rowptr.p, d_perm.p, d_c2c.p, C.coefnbr,
                C.d_fill_dst.p, C.d_wgt.p, d_key.p, d_slot.p, d_colof.p, d_bad.p};
    if (n > 0) k_spm_maps<<<cdiv(n * 32, 256), 256, 0, s>>>(C.meta, sm);
    // stable sort of the slots by permuted row (rows < n, absent mirrors = n)
    int bits = 1;
    while (((int64_t)1 << bits) <= n) bits++;
    size_t tmp_bytes = 0;
    PGPU_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_key.p, d_skey.p, d_slot.p, d_sslot.p,
                                               (int)(2 * nnz), 0, bits, s));
    PGPU_CHECK(d_tmp.alloc(std::max<size_t>(tmp_bytes, 1)));
    PGPU_CHECK(cub::DeviceRadixSort::SortPairs(d_tmp.p, tmp_bytes, d_key.p, d_skey.p, d_slot.p, d_sslot.p,
                                               (int)(2 * nnz), 0, bits, s));
    PGPU_CHECK(C.d_csr_ptr.alloc(n + 1));
    k_spm_rowptr<<<std::max(1, std::min(4096, cdiv(n + 1, 256))), 256, 0, s>>>((int)n, 2 * nnz, d_skey.p,
                                                                               C.d_csr_ptr.p);
    int64_t fnnz = 0;
    int bad = 0;
    PGPU_CHECK(cudaMemcpyAsync(&fnnz, C.d_csr_ptr.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    PGPU_CHECK(cudaMemcpyAsync(&bad, d_bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    if (bad) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(C.d_csr_col.alloc(std::max<int64_t>(fnnz, 1)));
    PGPU_CHECK(C.d_csr_src.alloc(std::max<int64_t>(fnnz, 1)));
    if (fnnz > 0)
        k_spm_csr<<<(int)std::min<int64_t>(4096, (fnnz + 255) / 256), 256, 0, s>>>(
            fnnz, d_sslot.p, d_colof.p, d_rowptr.p, herm ? 1 : 0, C.d_csr_col.p, C.d_csr_src.p);
    const int ncomp = (flttype == PGPU_COMPLEX64) ? 2 : 1;
    C.csr_nnz = fnnz;
    PGPU_CHECK(C.d_csr_val.alloc(std::max<int64_t>(fnnz, 1) * ncomp));
    PGPU_CHECK(C.d_vals.alloc(std::max<int64_t>(nnz, 1) * ncomp));
    PGPU_CHECK(cudaEventRecord(C.ev[5], s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[4], C.ev[5]));
    C.stats[15] = ms;   // device time of the pattern setup (uploads, maps, sort)
    C.have_spm = true;
    C.fact_done = -1;
    return PASTIX_GPU_SUCCESS;
}

static const int SMEM_LIMIT = 227 * 1024;   // opt-in shared memory per CTA
static const int WP_SMEM_LIMIT = SMEM_LIMIT - 1024;   // k_panel_wide's dynamic part (it has static arrays)

// --------------------------------------------------------------------------
// Factorization plan for one factorization type.
// --------------------------------------------------------------------------
// Off-diagonal rows of cblks taller than fuse_rows are solved by
// k_trsm_rows; shorter panels are factorized whole by k_panel_factor (the
// bound keeps the panel's shared-memory staging under the 227 KB limit for
// the element size).
static int fuse_rows_for(bool lu, size_t esz) {
    if (esz <= 4) return lu ? 256 : 1024;
    if (esz <= 8) return lu ? 96 : 512;
    return lu ? 48 : 256;
}
static const int TRSM_TR = 32;   // panel rows per k_trsm_rows CTA

// Single-precision update GEMMs large enough for a 128 x 128 tensor-core tile
// go to the tcgen05 kernel.  Tuning PGPU_TUNE_MIXED_GEMM selects the operand
// mode: 3xFP16 (default; per-row power-of-two scaled FP16 hi/lo split, about
// FP32 accuracy), 3xTF32 (the same split in TF32), TF32 (one product) or FP32
// (no tensor cores: FMA tiles only); its default comes from
// PASTIX_GPU_MIXED_GEMM = 3xf16 | 3xtf32 | tf32 | fp32.  The other knobs and their
// environment defaults: PGPU_TUNE_TC_KERNEL (PASTIX_GPU_TC_KERNEL=tile: one
// tile per CTA instead of the persistent kernel), PGPU_TUNE_LOOKAHEAD
// (PASTIX_GPU_LOOKAHEAD=0 disables it), PGPU_TUNE_LA_RESERVED_SMS (16),
// PGPU_TUNE_TRSM_GEMM (PASTIX_GPU_TRSM=rows disables the TRSM-as-GEMM path),
// PGPU_TUNE_TRSM_GEMM_ROWS (256: panels taller than this take it),
// PGPU_TUNE_TC_MIN_MN (8192: smallest M x N sent to the tensor cores).
enum { MG_FP32 = 0, MG_TF32 = 1, MG_3XTF32 = 2, MG_3XF16 = 3 };
static void default_tuning(int64_t *t) {
    const char *e = getenv("PASTIX_GPU_MIXED_GEMM");
    t[PGPU_TUNE_MIXED_GEMM] = (e && std::strcmp(e, "fp32") == 0)      ? MG_FP32
                              : (e && std::strcmp(e, "tf32") == 0)    ? MG_TF32
                              : (e && std::strcmp(e, "3xtf32") == 0) ? MG_3XTF32
                                                                      : MG_3XF16;
    e = getenv("PASTIX_GPU_TC_KERNEL");
    t[PGPU_TUNE_TC_KERNEL] = (e && std::strcmp(e, "tile") == 0) ? 0 : 1;
    e = getenv("PASTIX_GPU_LOOKAHEAD");
    t[PGPU_TUNE_LOOKAHEAD] = (e && std::strcmp(e, "0") == 0) ? 0 : 1;
    t[PGPU_TUNE_LA_RESERVED_SMS] = 16;
    e = getenv("PASTIX_GPU_TRSM");
    t[PGPU_TUNE_TRSM_GEMM] = (e && std::strcmp(e, "rows") == 0) ? 0 : 1;
    t[PGPU_TUNE_TRSM_GEMM_ROWS] = 256;
    t[PGPU_TUNE_TC_MIN_MN] = 128 * 64;
    e = getenv("PASTIX_GPU_WIDE_PANEL");
    t[PGPU_TUNE_WIDE_PANEL] = e ? std::atoi(e) : 128;
    e = getenv("PASTIX_GPU_TC_TMA");
    t[PGPU_TUNE_TC_TMA] = (e && std::strcmp(e, "0") == 0) ? 0 : 1;
    t[PGPU_TUNE_TC_PAIR_MIN] = -1;
    e = getenv("PASTIX_GPU_DMMA");
    t[PGPU_TUNE_DMMA] = (e && std::strcmp(e, "0") == 0) ? 0 : 1;
    e = getenv("PASTIX_GPU_SOLVE_FLOW");
    t[PGPU_TUNE_SOLVE_FLOW] = (e && std::strcmp(e, "0") == 0) ? 0 : 1;
    e = getenv("PASTIX_GPU_GRAPH");
    t[PGPU_TUNE_GRAPH] = e ? (std::strcmp(e, "1") == 0 ? 1 : 0) : -1;
}
static int mixed_gemm_mode(const pastix_gpu_t &C) { return (int)C.tune[PGPU_TUNE_MIXED_GEMM]; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); nullptr when the driver does not provide it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3-D map {K = w, rows, planes} over float rows of stride ld (elements),
// planes `plane` elements apart, box {32, 128, planes}, SWIZZLE_128B.
static bool encode_panel_map(CUtensorMap *map, float *base, int w, int rows, int ld, int planes, int64_t plane) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)w, (cuuint64_t)rows, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)std::max<int64_t>(plane, 1) * 4};
    const cuuint32_t box[3] = {(cuuint32_t)TC_BK, (cuuint32_t)TC_BM, (cuuint32_t)planes};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
// 3-D map {K = w, rows, 2 planes} over FP16 rows of ld16 halves, box
// {64, 128, 2} (128-byte rows, SWIZZLE_128B): one box lands the hi and the lo
// tile of a k-block.
static bool encode_h16_map(CUtensorMap *map, __half *base, int w, int rows, int ld16, int64_t plane) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)w, (cuuint64_t)rows, 2};
    const cuuint64_t strides[2] = {(cuuint64_t)ld16 * 2, (cuuint64_t)plane * 2};
    const cuuint32_t box[3] = {64, (cuuint32_t)TC_BM, 2};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
static bool tc_enabled(const pastix_gpu_t &C) { return mixed_gemm_mode(C) != MG_FP32; }
static bool tc_task(const pastix_gpu_t &C, int M, int N, int K) {
    return K >= 32 && M >= 64 && N >= 32 && (int64_t)M * N >= C.tune[PGPU_TUNE_TC_MIN_MN];
}

// Kernel form of a factorization request (pastix_factotype_t on a real or
// complex matrix): the real LDL^h is the LDL^t, LL^t of a complex symmetric
// matrix (PXTRF) is not provided.  -1 when unsupported.
static int fact_mode_of(int fact, bool zc) {
    switch (fact) {
    case PGPU_FACT_POTRF: return FM_POTRF;
    case PGPU_FACT_GETRF: return FM_GETRF;
    case PGPU_FACT_SYTRF: return FM_SYTRF;
    case PGPU_FACT_HETRF: return zc ? FM_HETRF : FM_SYTRF;
    case 3: return zc ? -1 : FM_POTRF;
    default: return -1;
    }
}


// Chunk width (bytes per row) of k_panel_wide for width w: the widest of
// 128 / 64 / 32 bytes whose buffers fit in shared memory, 0 if none does.
static int wide_kcb(int w, size_t esz, bool lu, bool ldl) {
    for (int kcb = 128; kcb >= 32; kcb /= 2)
        if (wp_smem_bytes(w, esz, lu, ldl, kcb) <= (size_t)WP_SMEM_LIMIT) return kcb;
    return 0;
}
// Diagonal blocks at least PGPU_TUNE_WIDE_PANEL columns wide (0: never)
// are factorized by k_panel_wide, when one CTA covers them (elements of up
// to 8 bytes).
static bool wide_panel(const pastix_gpu_t &C, int w, size_t esz, bool lu, bool ldl) {
    const int64_t wmin = C.tune[PGPU_TUNE_WIDE_PANEL];
    return wmin > 0 && w >= wmin && esz <= 8 && wp_tiles_fit(w, lu) && wide_kcb(w, esz, lu, ldl) > 0;
}

// Forget the captured factorization graph (its nodes name the plan's and the
// matrix's device buffers): called whenever those are rebuilt.
static void invalidate_graph(pastix_gpu_t &C) {
    if (C.fact_exec) cudaGraphExecDestroy(C.fact_exec);
    if (C.fact_graph) cudaGraphDestroy(C.fact_graph);
    C.fact_exec = nullptr;
    C.fact_graph = nullptr;
    for (int k = 0; k < 5; k++) C.graph_key[k] = -1;
}

// Clears the dataflow solve's counters, ticket counters, error flag and Z
// (a new plan, or a solve whose waits gave up).
static int flow_reset(pastix_gpu_t &C) {
    if (C.d_flow_cnt.n) PGPU_CHECK(cudaMemsetAsync(C.d_flow_cnt.p, 0, C.d_flow_cnt.n * sizeof(unsigned long long), C.stream));
    if (C.d_flowZ.n) PGPU_CHECK(cudaMemsetAsync(C.d_flowZ.p, 0, C.d_flowZ.n, C.stream));
    PGPU_CHECK(cudaMemsetAsync(C.d_flow_state.p, 0, sizeof(FlowState), C.stream));
    for (int d = 0; d < 2; d++) C.flow_epoch[d].assign(C.flow_runs.size(), 0);
    return PASTIX_GPU_SUCCESS;
}

// Runs of consecutive levels the dataflow solve takes (k_solve_flow): levels
// that are not solved one warp per cblk and whose cblks all hold the inverse
// of their diagonal block (and narrow enough for one stage's vector part of
// FLOW_MAXRHS right-hand sides, complex128: 2).  Tasks of at most
// FLOW_MAXROWS rows (fewer where a row is long: one staging buffer), in two
// lists per direction -- critical: the diagonal tasks and the updates of a
// cblk of the next level; the others -- each sorted by one key that is a
// dependency order (a task waits only for tasks with smaller keys):
//   forward, by deadline: D(c): 2 lev(c); O(c, f): 2 lev(f) - 1 (just before
//            D(f)), or 2 lb when f lies above the run; older sources first;
//   backward, by the point where the input exists, with depth
//            d = (last level of the run) - lev:  E(c): 2 d(c) + 1;
//            G(c, f): 2 d(f) + 2 (after x_f), or 0 when f lies above the run;
//            the nearest source first.
// (Forward, the deadline order keeps each level's inputs together; backward,
// the input order lets gathers run as soon as x_f exists: each measured the
// faster for its direction.)  Each record carries the task's deadline -- the
// key of the task that needs it (backward G: 2 d(c)) -- by which the fetch
// warp chooses between the heads of its two lists.  List task i goes to CTA
// i mod G (G: one CTA per SM); the lists are stored CTA by CTA.  Y and Z for
// up to FLOW_MAXRHS right-hand sides are allocated here, with the plan (the
// allocation-free solve allocates nothing).
static int build_flow_plan(pastix_gpu_t &C, size_t esz, bool lu) {
    C.flow_runs.clear();
    C.flow_maxw = 0;
    if (!C.trsm_gemm) return PASTIX_GPU_SUCCESS;
    const int nc = C.cblknbr;
    std::vector<char> ok(C.nlevels, 0);
    for (int l = 0; l < C.nlevels; l++) {
        bool all = !(C.lvl_maxw[l] <= 32 && C.lvl_maxh[l] <= SOLVE_SMALL_MAXH) && C.lvl_ptr[l + 1] > C.lvl_ptr[l];
        for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1] && all; q++) {
            const int c = C.lvl_cblks[q];
            const size_t vmax = (size_t)std::max(C.width[c], FLOW_MAXROWS) * (esz <= 8 ? FLOW_MAXRHS : 2) * esz;
            all = C.invoff[c] >= 0 && vmax + 16 <= (size_t)FLOW_VEC_BYTES && (size_t)C.ld[c] * esz <= (size_t)FLOW_STAGE;
        }
        ok[l] = all;
    }
    for (int l = 0; l < C.nlevels;) {
        if (!ok[l]) {
            l++;
            continue;
        }
        int e = l;
        while (e < C.nlevels && ok[e]) e++;
        C.flow_runs.push_back(make_int2(l, e));
        l = e;
    }
    if (C.flow_runs.empty()) return PASTIX_GPU_SUCCESS;
    std::vector<int> runid(nc, -1);
    for (size_t r = 0; r < C.flow_runs.size(); r++)
        for (int q = C.lvl_ptr[C.flow_runs[r].x]; q < C.lvl_ptr[C.flow_runs[r].y]; q++) {
            runid[C.lvl_cblks[q]] = (int)r;
            C.flow_maxw = std::max(C.flow_maxw, C.width[C.lvl_cblks[q]]);
        }
    std::vector<int> need(4 * (size_t)nc, 0);   // nd, noin, ngo, ned
    int G = 0;   // CTAs of a launch: one per SM
    PGPU_CHECK(cudaDeviceGetAttribute(&G, cudaDevAttrMultiProcessorCount, C.device));
    int *nd = need.data(), *noin = nd + nc, *ngo = noin + nc, *ned = ngo + nc;
    C.flow_G = G;
    std::vector<FlowTask> all[2];
    std::vector<int> offs[2];
    for (int d = 0; d < 2; d++) C.flow_tptr[d].assign(1, 0);
    for (size_t r = 0; r < C.flow_runs.size(); r++) {
        const int la = C.flow_runs[r].x, lb = C.flow_runs[r].y;
        auto lev = [&](int c) { return C.cblk_level[c]; };
        // the factor rows of a task: D / E rows of the inverse (forward LU: the
        // second, unit-lower one), O / G rows of the panel (backward LU: U^t)
        auto task = [&](int kind, bool fwd, int flag, int nr, int c, int r0, int f) {
            FlowTask t;
            t.hdr = kind | (flag << 3) | (nr << 4);
            t.c = c;
            t.r0 = r0;
            t.f = f;
            t.w = C.width[c];
            t.ld = C.ld[c];
            t.fc = C.fcol[c];
            t.need = 0;   // (set once every task of the run is counted)
            if (kind == FLOW_D) {
                t.src = C.invoff[c] + (fwd && lu ? inv_span(C.width[c], C.ld[c]) : 0) + (int64_t)r0 * C.ld[c];
                t.aux = C.coefoff[c];
            } else {
                t.src = (!fwd && lu ? C.coefnbr : 0) + C.coefoff[c] + (int64_t)r0 * C.ld[c];
                t.aux = C.rowbase[c] + r0;
            }
            return t;
        };
        struct Keyed {
            int key, sec, seq;   // list order: key, then sec, then creation
            FlowTask t;
            bool high;           // critical list
            int deadline;        // the key of the task that needs it (stored in the record)
        };
        std::vector<Keyed> fw, bw;
        for (int l = la; l < lb; l++)
            for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1]; q++) {
                const int c = C.lvl_cblks[q];
                const int w = C.width[c];
                const int R = std::max(1, std::min(FLOW_MAXROWS, (int)((size_t)FLOW_STAGE / ((size_t)C.ld[c] * esz))));
                const int dc = lb - 1 - l;
                for (int n0 = 0; n0 < w; n0 += R) {
                    const int nr = std::min(R, w - n0);
                    fw.push_back({2 * l, 0, (int)fw.size(), task(FLOW_D, true, 0, nr, c, n0, 0), true, 2 * l});
                    bw.push_back({2 * dc + 1, 0, (int)bw.size(), task(FLOW_D, false, 0, nr, c, n0, 0), true,
                                  2 * dc + 1});
                    nd[c]++;
                    ned[c]++;
                }
                // off-diagonal rows, in runs of blocks facing the same cblk
                for (int b = C.fblok[c] + 1; b < C.fblok[c + 1];) {
                    const int f = C.bfcblk[b];
                    int e = b;
                    while (e < C.fblok[c + 1] && C.bfcblk[e] == f) e++;
                    const int ra = C.browoff[b], rb = C.browoff[e - 1] + C.blrow[e - 1] - C.bfrow[e - 1] + 1;
                    const bool in = runid[f] == (int)r;
                    const bool next = in && lev(f) == l + 1;
                    const int df = lb - 1 - lev(f);
                    for (int r0 = ra; r0 < rb; r0 += R) {
                        const int nr = std::min(R, rb - r0);
                        const int fkey = in ? 2 * lev(f) - 1 : 2 * lb;
                        fw.push_back({fkey, l, (int)fw.size(), task(FLOW_O, true, in ? 1 : 0, nr, c, r0, f), next, fkey});
                        bw.push_back({in ? 2 * df + 2 : 0, dc, (int)bw.size(),
                                      task(FLOW_O, false, in ? 1 : 0, nr, c, r0, f), next, 2 * dc});
                        if (in) noin[f]++;
                        ngo[c]++;
                    }
                    b = e;
                }
            }
        for (int d = 0; d < 2; d++) {
            std::vector<Keyed> &v = d ? bw : fw;
            std::stable_sort(v.begin(), v.end(), [](const Keyed &x, const Keyed &y) {
                if (x.high != y.high) return x.high;   // critical list first
                return x.key != y.key ? x.key < y.key : (x.sec != y.sec ? x.sec < y.sec : x.seq < y.seq);
            });
            int nh = 0;
            for (const Keyed &k : v) nh += k.high ? 1 : 0;
            // each list CTA by CTA: list task i goes to CTA i mod G, the CTA's tasks contiguous and in
            // list order; offsets: G + 1 for the critical list, then G + 1 for the other
            for (int part = 0; part < 2; part++) {
                const int b = part ? nh : 0, n = part ? (int)v.size() - nh : nh;
                offs[d].push_back(part ? nh : 0);
                for (int q = 0; q < G; q++) {
                    for (int i = q; i < n; i += G) {
                        FlowTask t = v[b + i].t;
                        const int kind = t.hdr & 7, flag = (t.hdr >> 3) & 1;
                        t.hdr |= v[b + i].deadline << 10;
                        if (d == 0) t.need = kind == FLOW_D ? noin[t.c] : nd[t.c];
                        else t.need = kind == FLOW_D ? ngo[t.c] : flag;
                        all[d].push_back(t);
                    }
                    offs[d].push_back((int)all[d].size() - C.flow_tptr[d].back());
                }
            }
            C.flow_tptr[d].push_back((int)all[d].size());
        }
    }
    for (int d = 0; d < 2; d++) PGPU_CHECK(C.d_flow_off[d].upload(offs[d], C.stream));
    for (int d = 0; d < 2; d++) PGPU_CHECK(C.d_flow_tasks[d].upload(all[d], C.stream));
    PGPU_CHECK(C.d_flow_need.upload(need, C.stream));
    if (C.d_flow_cnt.n < 5 * (size_t)nc) {
        C.d_flow_cnt.release();
        PGPU_CHECK(C.d_flow_cnt.alloc(5 * (size_t)nc));
    }
    const size_t vbytes = (size_t)C.n * FLOW_MAXRHS * esz;
    if (C.d_flowY.n < vbytes) {
        C.d_flowY.release();
        PGPU_CHECK(C.d_flowY.alloc(vbytes));
    }
    if (C.d_flowZ.n < vbytes) {
        C.d_flowZ.release();
        PGPU_CHECK(C.d_flowZ.alloc(vbytes));
    }
    return flow_reset(C);
}

static int build_fact_plan(pastix_gpu_t &C, int fmode, bool fp32, bool zc) {
    const bool use_tc = fp32 && !zc && tc_enabled(C) && (fmode == FM_POTRF || fmode == FM_GETRF);
    // real FP64: the large update and TRSM GEMMs on the FP64 tensor cores (DMMA),
    // planned like the single-precision tensor-core tiles (128 x 64 tiles)
    const bool use_dmma = !fp32 && !zc && C.tune[PGPU_TUNE_DMMA] != 0 && !C.record;
    // tile shape of the tensor-core lists: tcgen05 tiles in single precision
    // (update tiles of LL^t / LU, and the TRSM tiles of every real form,
    // LDL^t included), DMMA tiles in FP64
    const int tbm = fp32 ? TC_BM : DG_BM, tbn = fp32 ? TC_BN : DG_BN;
    const bool lu = (fmode == FM_GETRF), ldl = fm_ldl(fmode);
    // panels taller than TRSM_GEMM_ROWS: inverse of the diagonal block, then the
    // off-diagonal rows times it as a GEMM (tensor cores in single precision)
    const bool tgemm = !C.record && C.tune[PGPU_TUNE_TRSM_GEMM] != 0;
    const int key = ((((fmode * 2 + (fp32 ? 1 : 0)) * 2 + (use_tc ? 1 : 0)) * 2 + (zc ? 1 : 0)) * 2 + (tgemm ? 1 : 0));
    // (set_tuning invalidates the plan, so the knobs need no place in the key)
    if (C.plan_fact == key) return PASTIX_GPU_SUCCESS;
    invalidate_graph(C);   // the launch lists and workspaces the graph names are rebuilt
    const size_t esz = (fp32 ? 4 : 8) * (zc ? 2 : 1);
    const int fuse = tgemm ? std::min((int)C.tune[PGPU_TUNE_TRSM_GEMM_ROWS], fuse_rows_for(lu, esz))
                           : fuse_rows_for(lu, esz);
    const bool tc_trsm = tgemm && ((fp32 && !zc && tc_enabled(C)) || use_dmma);
    std::vector<int2> invjobs;
    std::vector<int4> ttiles, tttiles;
    int64_t inv_elems = 0, scr_max = 0;
    C.inv_ptr.assign(C.nlevels + 1, 0);
    C.ttile_ptr.assign(C.nlevels + 1, 0);
    C.tttile_ptr.assign(C.nlevels + 1, 0);
    C.invoff.assign(C.cblknbr, -1);
    C.scroff.assign(C.cblknbr, 0);
    const int sym_flags = 8 | (ldl ? 16 : 0) | ((zc && fm_conj(fmode)) ? 32 : 0);
    const double fma_flops = zc ? 8.0 : 2.0;
    std::vector<int4> tiles, trsm, tctiles;
    std::vector<GemmTask> tasks;
    double gflops = 0, tcflops = 0;
    C.tile_ptr.assign(C.nlevels + 1, 0);
    C.tctile_ptr.assign(C.nlevels + 1, 0);
    C.trsm_ptr.assign(C.nlevels + 1, 0);
    C.lvl_plrows.assign(C.nlevels, 0);
    C.lvl_porows.assign(C.nlevels, 0);
    C.lvl_pmaxw.assign(C.nlevels, 0);
    C.lvl_wmaxw.assign(C.nlevels, 0);
    C.pn_ptr.assign(C.nlevels + 1, 0);
    C.pw_ptr.assign(C.nlevels + 1, 0);
    std::vector<int2> pjobs, wjobs, sjobs;
    C.ps_ptr.assign(C.nlevels + 1, 0);
    C.tile_crit.assign(C.nlevels, 0);
    C.tctile_crit.assign(C.nlevels, 0);
    std::vector<int4> lt[2], ltc[2], lsm[2];   // this level's FMA (CTA / warp) and tensor-core tiles: [0] next-level targets, [1] others
    // warp tiles for narrow FMA updates (not while recording task timings:
    // those describe the CTA tiles)
    const bool small_ok = !C.record && esz <= 8;
    C.stile_n.assign(2 * C.nlevels, 0);
    for (int l = 0; l < C.nlevels; l++) {
        int64_t scr_lvl = 0;
        for (int k = 0; k < 2; k++) {
            lt[k].clear();
            ltc[k].clear();
        }
        for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1]; q++) {
            const int c = C.lvl_cblks[q];
            const int w = C.width[c], h = C.height[c];
            const int rows = (h <= fuse) ? h : w;
            if (rows == w && wide_panel(C, w, esz, lu, ldl)) {
                wjobs.push_back(make_int2(c, q));
                C.lvl_wmaxw[l] = std::max(C.lvl_wmaxw[l], w);
            } else if (w <= PB && esz <= 8 && !C.record) {
                sjobs.push_back(make_int2(c, q));   // one 32-column tile: one warp
            } else {
                pjobs.push_back(make_int2(c, q));
                C.lvl_plrows[l] = std::max(C.lvl_plrows[l], rows);
                C.lvl_porows[l] = std::max(C.lvl_porows[l], rows - w);
                C.lvl_pmaxw[l] = std::max(C.lvl_pmaxw[l], w);
            }
            if (h > fuse)
                for (int r0 = w; r0 < h; r0 += TRSM_TR) {
                    trsm.push_back(make_int4(c, r0, 0, lu ? 1 : (ldl ? 3 : 0)));
                    if (lu) trsm.push_back(make_int4(c, r0, 1, 2));
                }
            if (h > fuse && h > w && tgemm) {
                // inverse of the diagonal block, then X = A_off B^t into the scratch
                // (LU: two inverses and two outputs, the L and the U^t side)
                const int sides = lu ? 2 : 1;
                C.invoff[c] = inv_elems;
                inv_elems += sides * inv_span(w, C.ld[c]);
                for (int kind = 0; kind < sides; kind++)
                    for (int jb = 0; jb < w; jb += PB) invjobs.push_back(make_int2(c, jb + (kind << 20)));
                C.scroff[c] = scr_lvl;
                scr_lvl += sides * inv_span(h - w, C.ld[c]);
                for (int side = 0; side < sides; side++) {
                    const int id = (int)tasks.size();
                    GemmTask g{c, C.fblok[c], c, w, h - w, side ? (64 | 128 | 1) : 64, 0};
                    g.out = C.scroff[c] + (side ? inv_span(h - w, C.ld[c]) : 0);
                    tasks.push_back(g);
                    const int bm = tc_trsm ? tbm : GEMM_TM, bn = tc_trsm ? tbn : GEMM_TN;
                    for (int tm = 0; tm < cdiv(h - w, bm); tm++)
                        for (int tn = 0; tn < cdiv(w, bn); tn++)
                            (tc_trsm ? tttiles : ttiles).push_back(make_int4(id, tm, tn, 0));
                }
            } else if (h > fuse && h == w && tgemm) {
                // a wide cblk without off-diagonal rows (a root): the inverse alone, for
                // the solve's products with it (no TRSM)
                const int sides = lu ? 2 : 1;
                C.invoff[c] = inv_elems;
                inv_elems += sides * inv_span(w, C.ld[c]);
                for (int kind = 0; kind < sides; kind++)
                    for (int jb = 0; jb < w; jb += PB) invjobs.push_back(make_int2(c, jb + (kind << 20)));
            }
            const int b1 = C.fblok[c + 1];
            for (int b = C.fblok[c] + 1; b < b1; b++) {
                const int f = C.bfcblk[b];
                const int N = C.blrow[b] - C.bfrow[b] + 1;
                const int crit = (C.cblk_level[f] == l + 1) ? 0 : 1;
                auto add = [&](int arow0, int flags) {
                    const int M = h - arow0;
                    if (M <= 0) return;
                    const int id = (int)tasks.size();
                    tasks.push_back(GemmTask{c, b, f, arow0, M, flags});
                    gflops += fma_flops * M * N * w;
                    if ((use_tc || use_dmma) && tc_task(C, M, N, w)) {
                        tcflops += 2.0 * M * N * w;
                        for (int tm = 0; tm < cdiv(M, tbm); tm++)
                            for (int tn = 0; tn < cdiv(N, tbn); tn++) {
                                if ((flags & 8) && (int64_t)(tm + 1) * tbm <= (int64_t)tn * tbn) continue;
                                ltc[crit].push_back(make_int4(id, tm, tn, 0));
                            }
                        return;
                    }
                    if (small_ok && N <= GS_TN) {   // narrow update: one warp per 32 rows
                        for (int tm = 0; tm < cdiv(M, GS_TM); tm++) lsm[crit].push_back(make_int4(id, tm, 0, 1));
                        return;
                    }
                    for (int tm = 0; tm < cdiv(M, GEMM_TM); tm++)
                        for (int tn = 0; tn < cdiv(N, GEMM_TN); tn++) {
                            if ((flags & 8) && tm < tn) continue;   // strictly upper tiles of the diagonal block
                            lt[crit].push_back(make_int4(id, tm, tn, 0));
                        }
                };
                if (!lu) {
                    add(C.browoff[b], sym_flags);
                } else {
                    add(C.browoff[b], 2);                          // L side: A = L, B = U^T rows of b
                    if (b + 1 < b1) add(C.browoff[b + 1], 1 | 4);  // U side: A = U^T, B = L rows of b
                }
            }
        }
        // each part: the CTA tiles, then the warp tiles (counted in stile_n)
        for (int k = 0; k < 2; k++) {
            C.stile_n[2 * l + k] = (int)lsm[k].size();
            lt[k].insert(lt[k].end(), lsm[k].begin(), lsm[k].end());
            lsm[k].clear();
        }
        C.tile_crit[l] = (int)lt[0].size();
        C.tctile_crit[l] = (int)ltc[0].size();
        for (int k = 0; k < 2; k++) {
            tiles.insert(tiles.end(), lt[k].begin(), lt[k].end());
            tctiles.insert(tctiles.end(), ltc[k].begin(), ltc[k].end());
        }
        C.tile_ptr[l + 1] = (int)tiles.size();
        C.tctile_ptr[l + 1] = (int)tctiles.size();
        C.trsm_ptr[l + 1] = (int)trsm.size();
        C.pn_ptr[l + 1] = (int)pjobs.size();
        C.ps_ptr[l + 1] = (int)sjobs.size();
        C.pw_ptr[l + 1] = (int)wjobs.size();
        C.inv_ptr[l + 1] = (int)invjobs.size();
        C.ttile_ptr[l + 1] = (int)ttiles.size();
        C.tttile_ptr[l + 1] = (int)tttiles.size();
        scr_max = std::max(scr_max, scr_lvl);
    }
    // TMA operands (3xTF32, persistent kernel): hi/lo mirrors, tensor maps of
    // the source cblks, split jobs of their off-diagonal rows per level
    C.tma = use_tc && (mixed_gemm_mode(C) == MG_3XTF32 || mixed_gemm_mode(C) == MG_3XF16) &&
            C.tune[PGPU_TUNE_TC_KERNEL] != 0 && !C.record &&
            C.tune[PGPU_TUNE_TC_TMA] != 0 && tensor_map_encoder() != nullptr;
    C.split_ptr.assign(C.nlevels + 1, 0);
    C.h16 = C.tma && mixed_gemm_mode(C) == MG_3XF16;
    std::vector<int> mapidx_h;        // operand maps of each source cblk (TMA modes), for the tile descriptors
    std::vector<int64_t> hsbase_h;
    if (C.h16) {
        // 3xFP16: FP16 planes and row scales of the source matrices only (the
        // panels and inverses that feed a tensor-core task), in level order
        std::vector<char> src(C.cblknbr, 0);
        for (const int4 &t : tctiles) src[tasks[t.x].c] = 1;
        for (const int4 &t : tttiles) src[tasks[t.x].c] = 1;
        std::vector<int> mapidx(C.cblknbr, -1);
        std::vector<int64_t> hoff, hsbase;
        int64_t hp = 0, sp = 0;
        auto needed = [&](int c, int kind) {
            return kind == TMAP_L || (kind == TMAP_U && lu) || (kind == TMAP_I && C.invoff[c] >= 0) ||
                   (kind == TMAP_I2 && lu && C.invoff[c] >= 0);
        };
        for (int l = 0; l < C.nlevels; l++)
            for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1]; q++) {
                const int c = C.lvl_cblks[q];
                if (!src[c]) continue;
                const int w = C.width[c];
                mapidx[c] = (int)hoff.size();
                for (int kind = 0; kind < TMAP_KINDS; kind++) {
                    const bool nd = needed(c, kind);
                    const int rows = kind < TMAP_I ? C.height[c] : w;
                    hoff.push_back(nd ? hp : -1);
                    hsbase.push_back(nd ? sp : -1);
                    if (nd) {
                        hp += round_up((int64_t)rows * ld16_of(w), 64);
                        sp += rows;
                    }
                }
            }
        C.h16_plane = round_up(std::max<int64_t>(hp, 64), 64);
        if (C.d_h16.n < (size_t)(2 * C.h16_plane)) PGPU_CHECK(C.d_h16.alloc(2 * C.h16_plane));
        if (C.d_hscale.n < (size_t)std::max<int64_t>(sp, 1)) PGPU_CHECK(C.d_hscale.alloc(std::max<int64_t>(sp, 1)));
        std::vector<CUtensorMap> maps(hoff.size());
        if (!maps.empty()) std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
        std::vector<int4> split;
        for (int l = 0; l < C.nlevels && C.tma; l++) {
            for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1]; q++) {
                const int c = C.lvl_cblks[q];
                if (mapidx[c] < 0) continue;
                const int w = C.width[c], h = C.height[c];
                for (int kind = 0; kind < TMAP_KINDS; kind++) {
                    const int mi = mapidx[c] + kind;
                    if (hoff[mi] < 0) continue;
                    const int rows = kind < TMAP_I ? h : w;
                    if (!encode_h16_map(&maps[mi], C.d_h16.p + hoff[mi], w, rows, ld16_of(w), C.h16_plane))
                        C.tma = false;
                    // panels: their off-diagonal rows; inverses: all rows
                    for (int r0 = kind < TMAP_I ? w : 0; r0 < rows; r0 += 32) split.push_back(make_int4(c, r0, kind, 0));
                }
            }
            C.split_ptr[l + 1] = (int)split.size();
        }
        if (C.tma) {
            PGPU_CHECK(C.d_tmaps.upload(maps, C.stream));
            PGPU_CHECK(C.d_mapidx.upload(mapidx, C.stream));
            PGPU_CHECK(C.d_split.upload(split, C.stream));
            PGPU_CHECK(C.d_hoff.upload(hoff, C.stream));
            PGPU_CHECK(C.d_hsbase.upload(hsbase, C.stream));
            mapidx_h.swap(mapidx);
            hsbase_h.swap(hsbase);
        } else {
            C.h16 = false;
            C.split_ptr.assign(C.nlevels + 1, 0);
        }
    } else if (C.tma) {
        std::vector<char> src(C.cblknbr, 0);
        for (const int4 &t : tctiles) src[tasks[t.x].c] = 1;
        for (const int4 &t : tttiles) src[tasks[t.x].c] = 1;
        const int64_t ncoef = C.coefnbr * (lu ? 2 : 1);
        C.hilo_plane = (ncoef + 31) / 32 * 32;
        C.ihilo_plane = (inv_elems + 31) / 32 * 32;
        if (C.d_hilo.n < (size_t)(2 * C.hilo_plane)) PGPU_CHECK(C.d_hilo.alloc(2 * C.hilo_plane));
        if (C.d_ihilo.n < (size_t)(2 * C.ihilo_plane))
            PGPU_CHECK(C.d_ihilo.alloc(2 * std::max<int64_t>(C.ihilo_plane, 32)));
        // the inverses' strict upper parts are never written: zero planes
        PGPU_CHECK(cudaMemsetAsync(C.d_ihilo.p, 0, C.d_ihilo.n * sizeof(float), C.stream));
        std::vector<int> mapidx(C.cblknbr, -1);
        std::vector<CUtensorMap> maps;
        std::vector<int4> split;
        for (int l = 0; l < C.nlevels && C.tma; l++) {
            for (int q = C.lvl_ptr[l]; q < C.lvl_ptr[l + 1]; q++) {
                const int c = C.lvl_cblks[q];
                if (!src[c]) continue;
                const int w = C.width[c], h = C.height[c], ld = C.ld[c];
                mapidx[c] = (int)maps.size();
                maps.resize(maps.size() + TMAP_KINDS);
                CUtensorMap *mp = &maps[mapidx[c]];
                std::memset(mp, 0, TMAP_KINDS * sizeof(CUtensorMap));
                bool ok = encode_panel_map(mp + TMAP_L, C.d_hilo.p + C.coefoff[c], w, h, ld, 2, C.hilo_plane);
                if (lu) ok = ok && encode_panel_map(mp + TMAP_U, C.d_hilo.p + C.coefnbr + C.coefoff[c], w, h, ld, 2,
                                                    C.hilo_plane);
                if (C.invoff[c] >= 0) {
                    ok = ok && encode_panel_map(mp + TMAP_I, C.d_ihilo.p + C.invoff[c], w, w, ld, 2, C.ihilo_plane);
                    if (lu)
                        ok = ok && encode_panel_map(mp + TMAP_I2, C.d_ihilo.p + C.invoff[c] + inv_span(w, ld), w, w,
                                                    ld, 2, C.ihilo_plane);
                }
                if (!ok) C.tma = false;
                for (int r0 = w; r0 < h; r0 += 32)
                    for (int panel = 0; panel < (lu ? 2 : 1); panel++) split.push_back(make_int4(c, r0, panel, 0));
            }
            C.split_ptr[l + 1] = (int)split.size();
        }
        if (C.tma) {
            PGPU_CHECK(C.d_tmaps.upload(maps, C.stream));
            PGPU_CHECK(C.d_mapidx.upload(mapidx, C.stream));
            mapidx_h = mapidx;
            PGPU_CHECK(C.d_split.upload(split, C.stream));
        } else {
            C.split_ptr.assign(C.nlevels + 1, 0);
        }
    }
    if (C.tma) {
        {
            // pairs of 128-row tiles (tm even, tm + 1) of one task and column block
            // share their B tile in the TMA kernel: one entry {task, tm, tn, 1}
            // (a launch with fewer tiles than two per SM keeps them single: pairs
            // would leave SMs idle)
            int nsm_plan = 148;
            PGPU_CHECK(cudaDeviceGetAttribute(&nsm_plan, cudaDevAttrMultiProcessorCount, C.device));
            const int64_t pmin = C.tune[PGPU_TUNE_TC_PAIR_MIN] >= 0 ? C.tune[PGPU_TUNE_TC_PAIR_MIN] : 2 * nsm_plan;
            auto pair_range = [pmin](const std::vector<int4> &in, int b, int e, std::vector<int4> &out) {
                if (e - b < pmin) {
                    for (int i = b; i < e; i++) out.push_back(make_int4(in[i].x, in[i].y, in[i].z, 0));
                    return;
                }
                auto key = [](int t, int tm, int tn) { return ((int64_t)t << 32) | ((int64_t)tm << 16) | tn; };
                std::unordered_map<int64_t, int> pos;
                for (int i = b; i < e; i++) pos[key(in[i].x, in[i].y, in[i].z)] = i;
                std::vector<char> used(std::max(0, e - b), 0);
                for (int i = b; i < e; i++) {
                    if (used[i - b]) continue;
                    const int4 t = in[i];
                    used[i - b] = 1;
                    if ((t.y & 1) == 0) {
                        auto it = pos.find(key(t.x, t.y + 1, t.z));
                        if (it != pos.end() && !used[it->second - b]) {
                            used[it->second - b] = 1;
                            out.push_back(make_int4(t.x, t.y, t.z, 1));
                            continue;
                        }
                    }
                    out.push_back(make_int4(t.x, t.y, t.z, 0));
                }
            };
            std::vector<int4> ptc, ptt;
            std::vector<int> tc_ptr(C.nlevels + 1, 0), tt_ptr(C.nlevels + 1, 0), tc_crit(C.nlevels, 0);
            for (int l = 0; l < C.nlevels; l++) {
                const int b0 = C.tctile_ptr[l], bc = b0 + C.tctile_crit[l], b1 = C.tctile_ptr[l + 1];
                pair_range(tctiles, b0, bc, ptc);
                tc_crit[l] = (int)ptc.size() - tc_ptr[l];
                pair_range(tctiles, bc, b1, ptc);
                tc_ptr[l + 1] = (int)ptc.size();
                pair_range(tttiles, C.tttile_ptr[l], C.tttile_ptr[l + 1], ptt);
                tt_ptr[l + 1] = (int)ptt.size();
            }
            tctiles.swap(ptc);
            tttiles.swap(ptt);
            C.tctile_ptr.swap(tc_ptr);
            C.tctile_crit.swap(tc_crit);
            C.tttile_ptr.swap(tt_ptr);
        }
    }
    if (tgemm) {
        PGPU_CHECK(C.d_invjobs.upload(invjobs, C.stream));
        PGPU_CHECK(C.d_ttiles.upload(ttiles, C.stream));
        PGPU_CHECK(C.d_tttiles.upload(tttiles, C.stream));
        PGPU_CHECK(C.d_scroff.upload(C.scroff, C.stream));
        if (C.d_inv.n < (size_t)inv_elems * esz) {
            C.d_inv.release();
            PGPU_CHECK(C.d_inv.alloc((size_t)inv_elems * esz));
        }
        if (inv_elems) PGPU_CHECK(cudaMemsetAsync(C.d_inv.p, 0, (size_t)inv_elems * esz, C.stream));
        if (C.d_scr.n < (size_t)scr_max * esz) {
            C.d_scr.release();
            PGPU_CHECK(C.d_scr.alloc((size_t)scr_max * esz));
        }
    }
    PGPU_CHECK(C.d_invoff.upload(C.invoff, C.stream));
    C.meta.invoff = C.d_invoff.p;
    C.trsm_gemm = tgemm;
    cudaStream_t s = C.stream;
    // every tensor-core tile must start inside its task (a tile past the task
    // would hand the MMA an empty or negative width)
    for (const std::vector<int4> *lst : {&tctiles, &tttiles})
        for (const int4 &t : *lst) {
            const GemmTask &g = tasks[t.x];
            const int N = (g.flags & 64) ? C.width[g.c] : C.blrow[g.b] - C.bfrow[g.b] + 1;
            if ((int64_t)t.y * tbm >= g.M || (int64_t)t.z * tbn >= N ||
                ((t.w & 1) && (int64_t)(t.y + 1) * tbm >= g.M)) {
                fprintf(stderr, "pastix_gpu: tensor-core tile outside its task (plan error)\n");
                return PASTIX_GPU_ERR_INTERNAL;
            }
        }
    PGPU_CHECK(C.d_tiles.upload(tiles, s));
    PGPU_CHECK(C.d_tctiles.upload(tctiles, s));
    PGPU_CHECK(C.d_trsm.upload(trsm, s));
    PGPU_CHECK(C.d_tasks.upload(tasks, s));
    if (C.tma || use_dmma) {
        // tensor-core tasks: target-row maps (built on the device) and scale bases
        std::vector<int64_t> taux(3 * tasks.size(), 0);
        std::vector<char> is_tc(tasks.size(), 0);
        for (const int4 &t : tctiles) is_tc[t.x] = 1;
        std::vector<int> tlist;
        int64_t rows = 0;
        for (size_t i = 0; i < tasks.size(); i++) {
            const GemmTask &g = tasks[i];
            const bool trsm = (g.flags & 64) != 0;
            if (is_tc[i] && !trsm) {
                taux[3 * i] = rows;
                rows += g.M;
                tlist.push_back((int)i);
            }
            if (C.h16 && (is_tc[i] || trsm) && mapidx_h[g.c] >= 0) {
                const int mb = mapidx_h[g.c];
                const int ka = (g.flags & 1) ? TMAP_U : TMAP_L;
                const int kb = trsm ? ((g.flags & 128) ? TMAP_I2 : TMAP_I) : ((g.flags & 2) ? TMAP_U : TMAP_L);
                taux[3 * i + 1] = hsbase_h[mb + ka] + g.arow0;
                taux[3 * i + 2] = hsbase_h[mb + kb] + (trsm ? 0 : C.browoff[g.b]);
            }
        }
        PGPU_CHECK(C.d_taux.upload(taux, s));
        if (C.tma) {
            // one descriptor per tensor-core tile (k_gemm_scatter_tc_tma reads no task tables)
            auto make_desc = [&](const int4 &t) {
                const GemmTask &g = tasks[t.x];
                const bool trsm = (g.flags & 64) != 0;
                const int c = g.c, w = C.width[c];
                const int N = trsm ? w : C.blrow[g.b] - C.bfrow[g.b] + 1;
                const int i0 = t.y * TC_BM, j0 = t.z * TC_BN;
                const int mb = mapidx_h[c];
                TcDesc d;
                std::memset(&d, 0, sizeof(d));
                d.mapa = mb + ((g.flags & 1) ? TMAP_U : TMAP_L);
                d.mapb = mb + (trsm ? ((g.flags & 128) ? TMAP_I2 : TMAP_I) : ((g.flags & 2) ? TMAP_U : TMAP_L));
                d.rowa = g.arow0 + i0;
                d.rowb = (trsm ? 0 : C.browoff[g.b]) + j0;
                d.nk = cdiv(w, C.h16 ? 64 : TC_BK);
                d.ncols = std::min(TC_BN, N - j0);
                d.pair = t.w & 1;
                d.flags = g.flags;
                d.mrows = g.M - i0;
                if (trsm) {
                    d.ldo = C.ld[c];
                    d.off = g.out + (int64_t)i0 * C.ld[c] + j0;
                } else {
                    const int f = g.f;
                    d.ldo = C.ld[f];
                    d.wf = C.width[f];
                    d.tcol = C.bfrow[g.b] + j0 - C.fcol[f];
                    d.off = ((g.flags & 4) ? C.coefnbr : 0) + C.coefoff[f];
                    d.rmap = taux[3 * (size_t)t.x] + i0;
                }
                if (C.h16) {
                    d.sa = taux[3 * (size_t)t.x + 1] + i0;
                    d.sb = taux[3 * (size_t)t.x + 2] + j0;
                }
                return d;
            };
            std::vector<TcDesc> dtc(tctiles.size()), dtt(tttiles.size());
            for (size_t i = 0; i < tctiles.size(); i++) dtc[i] = make_desc(tctiles[i]);
            for (size_t i = 0; i < tttiles.size(); i++) dtt[i] = make_desc(tttiles[i]);
            PGPU_CHECK(C.d_tcdesc.upload(dtc, s));
            PGPU_CHECK(C.d_ttdesc.upload(dtt, s));
        }
        PGPU_CHECK(C.d_tlist.upload(tlist, s));
        if (C.d_tmap.n < (size_t)std::max<int64_t>(rows, 1)) PGPU_CHECK(C.d_tmap.alloc(std::max<int64_t>(rows, 1)));
        if (!tlist.empty())
            k_task_rowmap<<<(int)tlist.size(), 256, 0, s>>>(C.meta, C.d_tasks.p, C.d_tlist.p, C.d_taux.p,
                                                            C.d_tmap.p);
        PGPU_CHECK(cudaGetLastError());
    }
    PGPU_CHECK(C.d_pjobs.upload(pjobs, s));
    PGPU_CHECK(C.d_sjobs.upload(sjobs, s));
    PGPU_CHECK(C.d_wjobs.upload(wjobs, s));
    {
        int rc = build_flow_plan(C, esz, lu);
        if (rc) return rc;
    }
    PGPU_CHECK(cudaStreamSynchronize(s));
    C.h_tiles.swap(tiles);
    C.h_tctiles.swap(tctiles);
    C.h_trsm.swap(trsm);
    C.h_tasks.swap(tasks);
    C.plan_fuse = fuse;
    C.plan_esz = (int)esz;
    C.plan_fmode = fmode;
    C.plan_fact = key;
    C.plan_gemm_flops = gflops;
    C.tc_flops = tcflops;
    return PASTIX_GPU_SUCCESS;
}

// Per-launch timing: one event recorded before every launch (and one after
// the last), so launch i took ev[i+1] - ev[i]; kinds[i] says which phase.
struct LaunchTimer {
    pastix_gpu_t &C;
    cudaStream_t st;
    std::vector<cudaEvent_t> &pool;
    std::vector<int> kinds, levels;   // per mark: phase kind, factorization level (-1 outside the level loop)
    int used = 0;
    int level = -1;
    explicit LaunchTimer(pastix_gpu_t &c) : C(c), st(c.stream), pool(c.evpool) {}
    LaunchTimer(pastix_gpu_t &c, cudaStream_t s, std::vector<cudaEvent_t> &p) : C(c), st(s), pool(p) {}
    // (inside a stream capture the record becomes an event node of the graph,
    // so a replay times its launches alike)
    cudaError_t mark(int kind) {
        if (used >= (int)pool.size()) {
            cudaEvent_t e;
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return r;
            pool.push_back(e);
        }
        kinds.push_back(kind);
        levels.push_back(level);
        // (in a capture a plain record only expresses a dependency; the
        // external form makes it an event-record node of the graph)
        return cudaEventRecordWithFlags(pool[used++], st, C.capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
    // after the stream was synchronized: accumulate ms per kind (a mark of
    // kind -1 closes an interval without opening a timed one)
    void collect(double *ms, int nkind) { collect_marks(pool, kinds, used, ms, nkind); }
    static void collect_marks(const std::vector<cudaEvent_t> &pool, const std::vector<int> &kinds, int used,
                              double *ms, int nkind) {
        for (int k = 0; k < nkind; k++) ms[k] = 0;
        for (int i = 0; i + 1 < used; i++) {
            float t = 0;
            if (kinds[i] >= 0 && kinds[i] < nkind && cudaEventElapsedTime(&t, pool[i], pool[i + 1]) == cudaSuccess)
                ms[kinds[i]] += t;
        }
    }
};

enum { PH_DIAG = 0, PH_TRSM = 1, PH_GEMM = 2, PH_TC = 3, PH_END = 4 };

template <typename T>
using PanelKernel = void (*)(Meta, const int2 *, T *, T *, const double *, int, int, int, Status *, int64_t *);
template <typename T>
using WideKernel = void (*)(Meta, const int2 *, T *, const double *, int, Status *, int64_t *);

template <typename T>
using SmallPanelKernel = void (*)(Meta, const int2 *, int, T *, T *, const double *, int, Status *);
template <typename T>
static SmallPanelKernel<T> panel_small_kernel(int fmode) {
    if constexpr (sizeof(T) > 8) {
        return nullptr;
    } else {
        switch (fmode) {
        case FM_GETRF: return k_panel_small<T, FM_GETRF>;
        case FM_SYTRF: return k_panel_small<T, FM_SYTRF>;
        case FM_HETRF:
            if constexpr (is_cplx<T>::value) return k_panel_small<T, FM_HETRF>;
            return nullptr;
        default: return k_panel_small<T, FM_POTRF>;
        }
    }
}

template <typename T>
static WideKernel<T> wide_kernel(int fmode) {
    if constexpr (sizeof(T) > 8) {
        return nullptr;
    } else {
        switch (fmode) {
        case FM_GETRF: return k_panel_wide<T, FM_GETRF>;
        case FM_SYTRF: return k_panel_wide<T, FM_SYTRF>;
        case FM_HETRF:
            if constexpr (is_cplx<T>::value) return k_panel_wide<T, FM_HETRF>;
            return nullptr;
        default: return k_panel_wide<T, FM_POTRF>;
        }
    }
}

template <typename T>
static PanelKernel<T> panel_kernel(int fmode) {
    switch (fmode) {
    case FM_GETRF: return k_panel_factor<T, FM_GETRF>;
    case FM_SYTRF: return k_panel_factor<T, FM_SYTRF>;
    case FM_HETRF:
        if constexpr (is_cplx<T>::value) return k_panel_factor<T, FM_HETRF>;
        return nullptr;
    default: return k_panel_factor<T, FM_POTRF>;
    }
}

// The hi / lo planes as the kernels' element type: only single-precision
// factors have them.
template <typename T>
static T *hilo_of(float *p) {
    if constexpr (std::is_same<T, float>::value) return p;
    else return nullptr;
}

template <typename T>
static int run_factor(pastix_gpu_t &C, int fmode, int *launches, LaunchTimer &tm) {
    const bool lu = (fmode == FM_GETRF);
    T *coefL = reinterpret_cast<T *>(C.d_coef.p);
    T *coefU = lu ? coefL + C.coefnbr : coefL;
    cudaStream_t s = C.stream;
    const int fuse = C.plan_fuse;   // rows the panel kernel solves itself (the plan's choice)
    PanelKernel<T> kpanel = panel_kernel<T>(fmode);
    if (!kpanel) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    if constexpr (sizeof(T) <= 8)
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_small<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        gs_smem_bytes<T>()));
    WideKernel<T> kwide = wide_kernel<T>(fmode);
    if (kwide)
        PGPU_CHECK(cudaFuncSetAttribute(kwide, cudaFuncAttributeMaxDynamicSharedMemorySize, WP_SMEM_LIMIT));
    // the Hermitian forms conjugate the L coefficients in the row solves
    constexpr bool CPX = is_cplx<T>::value;
    auto ktrsm = (CPX && fm_conj(fmode)) ? k_trsm_rows<T, TRSM_TR, CPX> : k_trsm_rows<T, TRSM_TR, false>;
    PGPU_CHECK(cudaFuncSetAttribute(kpanel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(ktrsm, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(k_tri_inverse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, WP_SMEM_LIMIT));
    // split products (3xTF32; the 3xFP16 mode without TMA operands falls back to it)
    const bool split = (mixed_gemm_mode(C) == MG_3XTF32 || mixed_gemm_mode(C) == MG_3XF16);
    const bool persist = C.tune[PGPU_TUNE_TC_KERNEL] != 0 && !C.record;   // task timings need one tile per CTA
    int nsm = 148;
    if constexpr (std::is_same<T, float>::value) {
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tc_smem_bytes<false>()));
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tc_smem_bytes<true>()));
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc_persistent<false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, tcp_smem_bytes<false>()));
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc_persistent<true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, tcp_smem_bytes<true>()));
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tma_smem_bytes<true>()));
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_tc_tma<true, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem_bytes<true>()));
        PGPU_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, C.device));
    }
    if constexpr (std::is_same<T, double>::value)
        PGPU_CHECK(cudaFuncSetAttribute(k_gemm_scatter_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        dg_smem_bytes()));
    int64_t *prof[4] = {nullptr, nullptr, nullptr, nullptr};
    if (C.record) {
        const size_t cnt[4] = {(size_t)C.cblknbr, (size_t)C.trsm_ptr[C.nlevels], (size_t)C.tile_ptr[C.nlevels],
                               (size_t)C.tctile_ptr[C.nlevels]};
        for (int k = 0; k < 4; k++) {
            if (C.d_prof[k].n < 2 * cnt[k]) PGPU_CHECK(C.d_prof[k].alloc(2 * cnt[k]));
            prof[k] = cnt[k] ? C.d_prof[k].p : nullptr;
        }
    }
    auto at = [](int64_t *p, int off) { return p ? p + 2 * (int64_t)off : nullptr; };
    const double *critp = C.d_fact_scal.p + 1;
    int nl = 0, ngemm = 0;
    // lookahead over two streams (off while recording task timings)
    const bool la = C.tune[PGPU_TUNE_LOOKAHEAD] != 0 && !C.record;
    LaunchTimer tm2(C, C.stream2, C.evpool2);
    if (la) {
        while ((int)C.la_events.size() < 2 * C.nlevels + 2) {
            cudaEvent_t e;
            PGPU_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            C.la_events.push_back(e);
        }
        // stream2 forks from the main stream after the fill-in
        PGPU_CHECK(cudaEventRecord(C.la_events[2 * C.nlevels], s));
        PGPU_CHECK(cudaStreamWaitEvent(C.stream2, C.la_events[2 * C.nlevels], 0));
    }
    // hi / lo split of the level's tensor-core source rows (before their first use as TMA operands)
    auto split_level = [&](int l) {
        if constexpr (std::is_same<T, float>::value) {
            const int nsp = C.split_ptr[l + 1] - C.split_ptr[l];
            if (C.tma && C.h16 && nsp) {
                k_split_rows_h16<<<nsp, 256, 0, s>>>(C.meta, C.d_split.p + C.split_ptr[l], coefL, coefU,
                                                     reinterpret_cast<const float *>(C.d_inv.p), C.d_h16.p,
                                                     C.h16_plane, C.d_hscale.p, C.d_hoff.p, C.d_hsbase.p,
                                                     C.d_mapidx.p);
                nl++;
            } else if (C.tma && nsp) {
                k_split_rows<<<nsp, 256, 0, s>>>(C.meta, C.d_split.p + C.split_ptr[l], coefL, coefU, C.d_hilo.p,
                                                 C.hilo_plane, C.coefnbr);
                nl++;
            }
        }
    };
    auto launch_gemms = [&](cudaStream_t st, LaunchTimer &lt, int t0, int nt, int nw, int c0, int ntc,
                            int gcap) -> int {
        // tiles [t0, t0 + nt): CTA tiles, then nw warp tiles
        if (nt - nw > 0) {
            PGPU_CHECK(lt.mark(PH_GEMM));
            k_gemm_scatter<T><<<nt - nw, 256, 0, st>>>(C.meta, C.d_tiles.p + t0, C.d_tasks.p, coefL, coefU, nullptr,
                                                       nullptr, at(prof[2], t0));
            if (la) PGPU_CHECK(lt.mark(PH_END));
            nl++;
            ngemm++;
        }
        if constexpr (sizeof(T) <= 8) {
            if (nw > 0) {
                PGPU_CHECK(lt.mark(PH_GEMM));
                k_gemm_scatter_small<T><<<cdiv(nw, GS_WARPS), GS_WARPS * 32, gs_smem_bytes<T>(), st>>>(
                    C.meta, C.d_tiles.p + t0 + nt - nw, nw, C.d_tasks.p, coefL, coefU);
                if (la) PGPU_CHECK(lt.mark(PH_END));
                nl++;
                ngemm++;
            }
        }
        if constexpr (std::is_same<T, double>::value) {
            if (ntc) {   // FP64 tensor cores (DMMA)
                PGPU_CHECK(lt.mark(PH_TC));
                k_gemm_scatter_dmma<<<ntc, DG_THREADS, dg_smem_bytes(), st>>>(
                    C.meta, C.d_tctiles.p + c0, C.d_tasks.p, coefL, coefU, nullptr, nullptr, C.d_tmap.p, C.d_taux.p);
                if (la) PGPU_CHECK(lt.mark(PH_END));
                nl++;
                ngemm++;
            }
        }
        if constexpr (std::is_same<T, float>::value) {
            if (ntc) {
                PGPU_CHECK(lt.mark(PH_TC));
                if (persist && C.tma && C.h16) {
                    const int g = std::min(ntc, gcap);
                    k_gemm_scatter_tc_tma<true, true><<<g, TMA_THREADS, tma_smem_bytes<true>(), st>>>(
                        C.d_tcdesc.p + c0, ntc, coefL, C.d_status.p, nullptr, C.d_tmaps.p, C.d_tmap.p,
                        C.d_hscale.p);
                } else if (persist && C.tma) {
                    const int g = std::min(ntc, gcap);
                    k_gemm_scatter_tc_tma<true><<<g, TMA_THREADS, tma_smem_bytes<true>(), st>>>(
                        C.d_tcdesc.p + c0, ntc, coefL, C.d_status.p, nullptr, C.d_tmaps.p, C.d_tmap.p);
                } else if (persist) {
                    const int g = std::min(ntc, gcap);
                    if (split)
                        k_gemm_scatter_tc_persistent<true><<<g, TCP_THREADS, tcp_smem_bytes<true>(), st>>>(
                            C.meta, C.d_tctiles.p + c0, ntc, C.d_tasks.p, coefL, coefU, C.d_status.p, nullptr,
                            nullptr);
                    else
                        k_gemm_scatter_tc_persistent<false><<<g, TCP_THREADS, tcp_smem_bytes<false>(), st>>>(
                            C.meta, C.d_tctiles.p + c0, ntc, C.d_tasks.p, coefL, coefU, C.d_status.p, nullptr,
                            nullptr);
                } else if (split) {
                    k_gemm_scatter_tc<true><<<ntc, TC_THREADS, tc_smem_bytes<true>(), st>>>(
                        C.meta, C.d_tctiles.p + c0, C.d_tasks.p, coefL, coefU, C.d_status.p, nullptr, nullptr,
                        at(prof[3], c0));
                } else {
                    k_gemm_scatter_tc<false><<<ntc, TC_THREADS, tc_smem_bytes<false>(), st>>>(
                        C.meta, C.d_tctiles.p + c0, C.d_tasks.p, coefL, coefU, C.d_status.p, nullptr, nullptr,
                        at(prof[3], c0));
                }
                if (la) PGPU_CHECK(lt.mark(PH_END));
                nl++;
                ngemm++;
            }
        }
        return PASTIX_GPU_SUCCESS;
    };
    for (int l = 0; l < C.nlevels; l++) {
        const int ncb = C.lvl_ptr[l + 1] - C.lvl_ptr[l];
        tm.level = tm2.level = l;
        // the deferred updates into this level's cblks were issued on stream2 two levels back or earlier
        if (la && l >= 2) {
            PGPU_CHECK(tm.mark(PH_END));
            PGPU_CHECK(cudaStreamWaitEvent(s, C.la_events[2 * (l - 2) + 1], 0));
        }
        const int mw = C.lvl_maxw[l];
        PGPU_CHECK(tm.mark(PH_DIAG));
        const int npw = C.pw_ptr[l + 1] - C.pw_ptr[l], npn = C.pn_ptr[l + 1] - C.pn_ptr[l];
        if (npw) {
            // wide diagonal blocks first: they are the level's longest panels
            const int wmw = C.lvl_wmaxw[l];
            const int kcb = wide_kcb(wmw, sizeof(T), lu, fm_ldl(fmode));
            if (!kwide || kcb == 0) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
            bool done = false;
            if constexpr (std::is_same<T, float>::value) {
                // single-precision LL^t / LDL^t: the lookahead form when its two block columns fit
                static const bool la_off = getenv("PASTIX_GPU_WIDE_LA") && std::strcmp(getenv("PASTIX_GPU_WIDE_LA"), "0") == 0;
                const size_t lsm = wpla_smem_bytes(wmw, fm_ldl(fmode));
                if (!la_off && (fmode == FM_POTRF || fmode == FM_SYTRF) && lsm <= (size_t)WP_SMEM_LIMIT &&
                    wp_row_groups(wmw) * 8 <= 2 * (WP_THREADS - 32)) {
                    auto kla = fmode == FM_POTRF ? k_panel_wide_la<FM_POTRF> : k_panel_wide_la<FM_SYTRF>;
                    PGPU_CHECK(cudaFuncSetAttribute(kla, cudaFuncAttributeMaxDynamicSharedMemorySize, WP_SMEM_LIMIT));
                    kla<<<npw, WP_THREADS, lsm, s>>>(C.meta, C.d_wjobs.p + C.pw_ptr[l], coefL, critp, C.d_status.p,
                                                     prof[0]);
                    done = true;
                }
            }
            if (!done)
                kwide<<<npw, WP_THREADS, wp_smem_bytes(wmw, sizeof(T), lu, fm_ldl(fmode), kcb), s>>>(
                    C.meta, C.d_wjobs.p + C.pw_ptr[l], coefL, critp, kcb / (int)sizeof(T), C.d_status.p, prof[0]);
            nl++;
        }
        if constexpr (sizeof(T) <= 8) {
            const int nps = C.ps_ptr[l + 1] - C.ps_ptr[l];
            if (nps) {
                auto ks = panel_small_kernel<T>(fmode);
                if (!ks) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
                PGPU_CHECK(cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, ps_smem_bytes<T>(fmode == FM_GETRF)));
                ks<<<cdiv(nps, PS_WARPS), PS_WARPS * 32, ps_smem_bytes<T>(fmode == FM_GETRF), s>>>(
                    C.meta, C.d_sjobs.p + C.ps_ptr[l], nps, coefL, coefU, critp, fuse, C.d_status.p);
                nl++;
            }
        }
        if (npn) {
            const int pmw = C.lvl_pmaxw[l];
            const int pl = C.lvl_plrows[l], pu = lu ? pmw : 0, po = lu ? C.lvl_porows[l] : 0;
            const size_t psm = (size_t)(PB * PBL + PB + (size_t)(pl + pu + po) * PBL) * sizeof(T);
            if (psm > (size_t)SMEM_LIMIT) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
            kpanel<<<npn, 256, psm, s>>>(C.meta, C.d_pjobs.p + C.pn_ptr[l], coefL, coefU, critp, fuse, pl, pu,
                                         C.d_status.p, prof[0]);
            nl++;
        }
        const int ntr = C.trsm_ptr[l + 1] - C.trsm_ptr[l];
        const int nij = C.inv_ptr[l + 1] - C.inv_ptr[l];
        // (a level of roots may hold inverses and no TRSM rows)
        const bool inv_block = (ntr || nij) && C.trsm_gemm;
        if (inv_block) {
            T *inv = reinterpret_cast<T *>(C.d_inv.p);
            T *scr = reinterpret_cast<T *>(C.d_scr.p);
            // X[w][33] + a 32-row strip of L, kch columns wide (as wide as fits, a multiple of 32)
            const size_t xs = tri_inverse_lb_offset(mw, sizeof(T));
            const int vk = std::max<int>(1, 16 / (int)sizeof(T));
            if (xs + (size_t)PB * (PB + vk) * sizeof(T) > (size_t)WP_SMEM_LIMIT) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
            int kch = (int)std::min<size_t>(round_up(mw, PB), ((WP_SMEM_LIMIT - xs) / ((size_t)PB * sizeof(T)) - vk));
            kch = std::max(PB, kch / PB * PB);
            size_t ism = xs + (size_t)PB * (kch + vk) * sizeof(T);
            // bulk-copied, double-buffered strips and tiles where they fit (rows of L; the U^t
            // columns of LU's first inverse keep the staged loads)
            const int slb = (int)round_up(mw, PB) + vk;
            const size_t bsm = xs + 2 * ((size_t)PB * slb + (size_t)PB * (PB + vk)) * sizeof(T);
            const int bulk_lb = bsm <= (size_t)WP_SMEM_LIMIT ? slb : 0;
            if (bulk_lb) ism = std::max(ism, bsm);
            PGPU_CHECK(tm.mark(PH_TRSM));
            k_tri_inverse<T><<<nij, 256, ism, s>>>(C.meta, C.d_invjobs.p + C.inv_ptr[l], coefL, inv,
                                                   fm_ldl(fmode) ? 1 : 0, (CPX && fm_conj(fmode)) ? 1 : 0,
                                                   fm_ldl(fmode) ? 1 : 0, lu ? 1 : 0, kch,
                                                   (C.tma && !C.h16) ? hilo_of<T>(C.d_ihilo.p) : nullptr,
                                                   C.ihilo_plane, bulk_lb, C.d_status.p);
            nl++;
            split_level(l);
            const int ntt = C.ttile_ptr[l + 1] - C.ttile_ptr[l];
            if (ntt) {
                k_gemm_scatter<T><<<ntt, 256, 0, s>>>(C.meta, C.d_ttiles.p + C.ttile_ptr[l], C.d_tasks.p, coefL, coefU,
                                                      inv, scr, nullptr);
                nl++;
            }
            if constexpr (std::is_same<T, double>::value) {
                const int ntc = C.tttile_ptr[l + 1] - C.tttile_ptr[l];
                if (ntc) {
                    k_gemm_scatter_dmma<<<ntc, DG_THREADS, dg_smem_bytes(), s>>>(
                        C.meta, C.d_tttiles.p + C.tttile_ptr[l], C.d_tasks.p, coefL, coefU, inv, scr, C.d_tmap.p,
                        C.d_taux.p);
                    nl++;
                }
            }
            if constexpr (std::is_same<T, float>::value) {
                const int ntc = C.tttile_ptr[l + 1] - C.tttile_ptr[l];
                if (ntc) {
                    const int g = std::min(ntc, nsm);
                    if (C.tma && C.h16)
                        k_gemm_scatter_tc_tma<true, true><<<g, TMA_THREADS, tma_smem_bytes<true>(), s>>>(
                            C.d_ttdesc.p + C.tttile_ptr[l], ntc, coefL, C.d_status.p, scr, C.d_tmaps.p, C.d_tmap.p,
                            C.d_hscale.p);
                    else if (C.tma)
                        k_gemm_scatter_tc_tma<true><<<g, TMA_THREADS, tma_smem_bytes<true>(), s>>>(
                            C.d_ttdesc.p + C.tttile_ptr[l], ntc, coefL, C.d_status.p, scr, C.d_tmaps.p, C.d_tmap.p);
                    else if (split)
                        k_gemm_scatter_tc_persistent<true><<<g, TCP_THREADS, tcp_smem_bytes<true>(), s>>>(
                            C.meta, C.d_tttiles.p + C.tttile_ptr[l], ntc, C.d_tasks.p, coefL, coefU, C.d_status.p,
                            inv, scr);
                    else
                        k_gemm_scatter_tc_persistent<false><<<g, TCP_THREADS, tcp_smem_bytes<false>(), s>>>(
                            C.meta, C.d_tttiles.p + C.tttile_ptr[l], ntc, C.d_tasks.p, coefL, coefU, C.d_status.p,
                            inv, scr);
                    nl++;
                }
            }
            bool copied = false;
            if constexpr (std::is_same<T, float>::value) {
                if (C.tma && C.h16) {
                    if (ntr)
                        k_trsm_copyback_h16<<<ntr, 256, 0, s>>>(C.meta, C.d_trsm.p + C.trsm_ptr[l], C.d_scroff.p,
                                                                scr, coefL, coefU, C.d_h16.p, C.h16_plane,
                                                                C.d_hscale.p, C.d_hoff.p, C.d_hsbase.p, C.d_mapidx.p);
                    copied = true;
                }
            }
            if (!copied && ntr)
                k_trsm_copyback<T><<<ntr, 256, 0, s>>>(C.meta, C.d_trsm.p + C.trsm_ptr[l], C.d_scroff.p, scr, coefL,
                                                       coefU, C.tma ? hilo_of<T>(C.d_hilo.p) : nullptr, C.hilo_plane,
                                                       C.coefnbr);
            if (ntr) nl++;
        } else if (ntr) {
            const size_t fixed = ((size_t)TRSM_TR * (mw + 1) + PB * PBL) * sizeof(T);
            const int pch = (int)std::min<size_t>(mw, (SMEM_LIMIT - std::min<size_t>(fixed, SMEM_LIMIT)) /
                                                          (PBL * sizeof(T)));
            if (pch < std::min(PB, mw)) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
            const size_t tsm = fixed + (size_t)pch * PBL * sizeof(T);
            PGPU_CHECK(tm.mark(PH_TRSM));
            ktrsm<<<ntr, 256, tsm, s>>>(C.meta, C.d_trsm.p + C.trsm_ptr[l], coefL, coefU, mw, pch,
                                        at(prof[1], C.trsm_ptr[l]));
            nl++;
        }
        if (!inv_block) split_level(l);   // the level's rows are final here
        // update GEMMs of the level: with lookahead the tiles whose target is
        // in the next level run here, the rest on stream2 once this level's
        // panels are final
        const int nti = C.tile_ptr[l + 1] - C.tile_ptr[l], ntc = C.tctile_ptr[l + 1] - C.tctile_ptr[l];
        if (la) {
            PGPU_CHECK(cudaEventRecord(C.la_events[2 * l], s));
            int rc = launch_gemms(s, tm, C.tile_ptr[l], C.tile_crit[l], C.stile_n[2 * l], C.tctile_ptr[l],
                                  C.tctile_crit[l], nsm);
            if (rc) return rc;
            PGPU_CHECK(cudaStreamWaitEvent(C.stream2, C.la_events[2 * l], 0));
            rc = launch_gemms(C.stream2, tm2, C.tile_ptr[l] + C.tile_crit[l], nti - C.tile_crit[l], C.stile_n[2 * l + 1],
                              C.tctile_ptr[l] + C.tctile_crit[l], ntc - C.tctile_crit[l],
                              std::max(1, nsm - (int)C.tune[PGPU_TUNE_LA_RESERVED_SMS]));
            if (rc) return rc;
            PGPU_CHECK(cudaEventRecord(C.la_events[2 * l + 1], C.stream2));
        } else {
            // (one launch per kind: the warp tiles of both parts sit at the parts' ends)
            int rc = launch_gemms(s, tm, C.tile_ptr[l], C.tile_crit[l], C.stile_n[2 * l], C.tctile_ptr[l], ntc, nsm);
            if (rc) return rc;
            rc = launch_gemms(s, tm, C.tile_ptr[l] + C.tile_crit[l], nti - C.tile_crit[l], C.stile_n[2 * l + 1], 0, 0,
                              nsm);
            if (rc) return rc;
        }
    }
    if (la && C.nlevels > 0) {
        // join the second stream after its last timing mark (which is itself a
        // graph node when the sequence is captured)
        PGPU_CHECK(tm2.mark(PH_END));
        PGPU_CHECK(cudaEventRecord(C.la_events[2 * C.nlevels + 1], C.stream2));
        PGPU_CHECK(cudaStreamWaitEvent(s, C.la_events[2 * C.nlevels + 1], 0));
    }
    PGPU_CHECK(tm.mark(PH_END));
    PGPU_CHECK(cudaGetLastError());
    // (the second stream's marks are read with the main stream's, after the
    // numfact, which ends on the main stream after it joined the second)
    if (C.capturing) {   // the replays collect the second stream's marks after their synchronization
        C.g_kinds2 = la ? tm2.kinds : std::vector<int>();
        C.g_used2 = la ? tm2.used : 0;
    }
    C.log_kinds2 = la ? tm2.kinds : std::vector<int>();
    C.log_levels2 = la ? tm2.levels : std::vector<int>();
    C.log_used2 = la ? tm2.used : 0;
    *launches = nl;
    C.stats[7] = ngemm;
    return PASTIX_GPU_SUCCESS;
}

// ||A||_F into d_fact_scal[0] and the static-pivot threshold into
// d_fact_scal[1], on the device (sopalin/pastix_task_sopalin.c:461-485; the
// bcsc stays double, so eps = dlamch('e') also for the mixed factors).
template <typename S>
static void dev_norm_and_crit(pastix_gpu_t &C, double magn) {
    cudaStream_t s = C.stream;
    const int nb = 512;
    k_sumsq_partial<S><<<nb, RED_THREADS, 0, s>>>(C.nnz, reinterpret_cast<const S *>(C.d_vals.p), C.d_wgt.p,
                                                  C.d_partial.p);
    k_dot_final<double><<<1, RED_THREADS, 0, s>>>(nb, C.d_partial.p, C.d_fact_scal.p, 1);
    k_static_pivot_threshold<<<1, 1, 0, s>>>(C.d_fact_scal.p, magn, 1.1102230246251565e-16);
}

// bcsc -> coeftab in the factor precision, then the level loop
template <typename T, typename S>
static int fill_and_factor(pastix_gpu_t &C, int fmode, int *nl, LaunchTimer &tm) {
    cudaStream_t s = C.stream;
    k_fillin<T, S><<<2048, 256, 0, s>>>(C.nnz, reinterpret_cast<const S *>(C.d_vals.p), C.d_fill_dst.p,
                                        reinterpret_cast<T *>(C.d_coef.p), C.d_status.p);
    return run_factor<T>(C, fmode, nl, tm);
}

// The last numfact's per-phase device times (stats 6, 8, 9, 11) and its
// phase timeline, from the timing events of both streams.  Called when they
// are first asked for rather than at the end of the numfact: reading a few
// hundred events costs about a millisecond of host time, which would
// otherwise sit between the factorization and the next call's launches.  The
// numfact's events (evpoolf, evpool2, ev[0]) are recorded only by numfact.
static void fact_marks_collect(pastix_gpu_t &C) {
    if (!C.fact_marks_pending) return;
    const bool replayed = C.fact_marks_pending == 2;
    C.fact_marks_pending = 0;
    if (replayed) LaunchTimer::collect_marks(C.evpool2, C.g_kinds2, C.g_used2, C.side_ms, 4);
    else LaunchTimer::collect_marks(C.evpool2, C.log_kinds2, C.log_used2, C.side_ms, 4);
    C.phase_info.clear();
    C.phase_times.clear();
    if (!replayed) {
        // both streams' marks on one timeline: elapsed time from the numfact's first event
        auto add = [&](int stream, const std::vector<cudaEvent_t> &pool, const std::vector<int> &kinds,
                       const std::vector<int> &levels, int used) {
            for (int i = 0; i + 1 < used; i++) {
                if (kinds[i] < 0 || kinds[i] >= PH_END) continue;   // PH_END closes an untimed gap
                float t0 = 0, t1 = 0;
                if (cudaEventElapsedTime(&t0, C.ev[0], pool[i]) != cudaSuccess ||
                    cudaEventElapsedTime(&t1, C.ev[0], pool[i + 1]) != cudaSuccess)
                    continue;
                C.phase_info.insert(C.phase_info.end(), {(int64_t)stream, (int64_t)kinds[i], (int64_t)levels[i]});
                C.phase_times.insert(C.phase_times.end(), {(double)t0, (double)t1});
            }
        };
        add(0, C.evpoolf, C.log_kinds, C.log_levels, C.log_used);
        add(1, C.evpool2, C.log_kinds2, C.log_levels2, C.log_used2);
    }
    double ph[4];
    if (replayed) LaunchTimer::collect_marks(C.evpoolf, C.g_kinds, C.g_used, ph, 4);
    else LaunchTimer::collect_marks(C.evpoolf, C.log_kinds, C.log_used, ph, 4);
    C.stats[8] = ph[PH_DIAG];
    C.stats[9] = ph[PH_TRSM];
    C.stats[6] = ph[PH_GEMM] + ph[PH_TC] + C.side_ms[PH_GEMM] + C.side_ms[PH_TC];
    C.stats[11] = ph[PH_TC] + C.side_ms[PH_TC];
}

extern "C" int pastix_gpu_numfact(pastix_gpu_t *ctx, const void *values) {
    if (!ctx || !values) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (!C.have_spm || C.cblknbr == 0) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(C.device));
    const int fact = (int)C.iparm[PGPU_IPARM_FACTORIZATION];
    const bool zc = (C.flttype == PGPU_COMPLEX64);
    const int fmode = fact_mode_of(fact, zc);
    if (fmode < 0) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    if (fmode != FM_GETRF && C.mtxtype == PGPU_GENERAL) return PASTIX_GPU_ERR_BADPARAMETER;
    const int mixed = C.iparm[PGPU_IPARM_MIXED] ? 1 : 0;
    int rc = build_fact_plan(C, fmode, mixed != 0, zc);
    if (rc) return rc;
    const size_t esz = (mixed ? 4 : 8) * (zc ? 2 : 1);
    const size_t vsz = zc ? 16 : 8;
    const size_t ncoef = (size_t)C.coefnbr * (fmode == FM_GETRF ? 2 : 1);
    if (C.d_coef.n < ncoef * esz) {
        C.d_coef.release();
        PGPU_CHECK(C.d_coef.alloc(ncoef * esz));
    }
    cudaStream_t s = C.stream;
    PGPU_CHECK(cudaEventRecord(C.ev[0], s));
    // values in (pastix_subtask_spm2bcsc), norm, bcsc -> coeftab
    PGPU_CHECK(cudaMemcpyAsync(C.d_vals.p, values, C.nnz * vsz,
                               is_device_ptr(values) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    int launches = 4;
    int nl = 0;
    C.fact_marks_pending = 0;
    LaunchTimer tm(C, s, C.evpoolf);
    auto enqueue = [&]() -> int {
        if (zc) dev_norm_and_crit<cdouble>(C, C.dparm[PGPU_DPARM_EPSILON_MAGN_CTRL]);
        else dev_norm_and_crit<double>(C, C.dparm[PGPU_DPARM_EPSILON_MAGN_CTRL]);
        if (zc)
            k_gather_vals<cdouble><<<1024, 256, 0, s>>>(C.csr_nnz, C.d_csr_src.p, (const cdouble *)C.d_vals.p,
                                                        (cdouble *)C.d_csr_val.p);
        else
            k_gather_vals<double><<<1024, 256, 0, s>>>(C.csr_nnz, C.d_csr_src.p, C.d_vals.p, C.d_csr_val.p);
        PGPU_CHECK(cudaMemsetAsync(C.d_status.p, 0, sizeof(Status), s));
        PGPU_CHECK(cudaMemsetAsync(C.d_coef.p, 0, ncoef * esz, s));
        if (zc)
            return mixed ? fill_and_factor<cfloat, cdouble>(C, fmode, &nl, tm)
                         : fill_and_factor<cdouble, cdouble>(C, fmode, &nl, tm);
        return mixed ? fill_and_factor<float, double>(C, fmode, &nl, tm)
                     : fill_and_factor<double, double>(C, fmode, &nl, tm);
    };
    // Graph replay (PGPU_TUNE_GRAPH): the sequence is captured once per
    // (plan, coeftab, mode, value buffer, pivot magnitude) as a CUDA graph and
    // replayed by later calls (the first call of a new plan captures,
    // instantiates and launches it).  The per-phase timings come from event
    // nodes of the graph.  Measured on one B200: the replay wins where the
    // launches outweigh the work (20^3 Laplacian: numfact 1.31 -> 1.23 ms,
    // time-to-solution end to end 2.54 -> 2.24 ms), is even on the 512 2D
    // systems (30.2 vs 30.6 ms) and loses on the large 3-D problems (80^3 LU:
    // 40.7 vs 44.2 ms); by default (-1) it is used for factors of at most
    // 2^24 coefficients.
    const int64_t gt = C.tune[PGPU_TUNE_GRAPH];
    const bool graph = !C.record && (gt == 1 || (gt < 0 && C.coefnbr <= ((int64_t)1 << 24)));
    bool replayed = false;
    if (graph) {
        int64_t magn_bits;   // the static-pivot magnitude is a kernel argument of the graph
        std::memcpy(&magn_bits, &C.dparm[PGPU_DPARM_EPSILON_MAGN_CTRL], sizeof(magn_bits));
        const int64_t key[5] = {C.plan_fact, (int64_t)(uintptr_t)C.d_coef.p, mixed * 8 + fmode,
                                (int64_t)(uintptr_t)C.d_vals.p, magn_bits};
        if (!C.fact_exec || std::memcmp(key, C.graph_key, sizeof(key)) != 0) {
            if (C.fact_exec) cudaGraphExecDestroy(C.fact_exec);
            if (C.fact_graph) cudaGraphDestroy(C.fact_graph);
            C.fact_exec = nullptr;
            C.fact_graph = nullptr;
            PGPU_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            C.capturing = true;
            rc = enqueue();
            C.capturing = false;
            C.g_kinds = tm.kinds;
            C.g_used = tm.used;
            C.g_nl = nl;
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(s, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            PGPU_CHECK(ec);
            C.fact_graph = g;
            PGPU_CHECK(cudaGraphInstantiate(&C.fact_exec, g, 0));
            std::memcpy(C.graph_key, key, sizeof(key));
        }
        PGPU_CHECK(cudaGraphLaunch(C.fact_exec, s));
        replayed = true;
    } else {
        rc = enqueue();
        if (rc) return rc;
    }
    PGPU_CHECK(cudaEventRecord(C.ev[1], s));
    Status st;
    double fscal[2];
    PGPU_CHECK(cudaMemcpyAsync(&st, C.d_status.p, sizeof(Status), cudaMemcpyDeviceToHost, s));
    PGPU_CHECK(cudaMemcpyAsync(fscal, C.d_fact_scal.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    C.dparm[PGPU_DPARM_A_NORM] = fscal[0];
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[0], C.ev[1]));
    C.stats[0] = launches + nl;
    C.stats[3] = ms;
    if (replayed) nl = C.g_nl;
    // per-phase times (stats 6, 8, 9, 11) and the timeline: read from the
    // events when first asked for (fact_marks_collect)
    C.log_kinds = tm.kinds;
    C.log_levels = tm.levels;
    C.log_used = tm.used;
    C.fact_marks_pending = replayed ? 2 : 1;
    C.stats[10] = C.plan_gemm_flops;
    C.stats[12] = C.tc_flops;   // tensor-core (tcgen05, or FP64 DMMA) task flops
    C.stats[13] = st.timeout;
    C.stats[14] = replayed ? 1.0 : 0.0;
    if (st.timeout || st.drain_timeout) {
        fprintf(stderr, "pastix_gpu: %d tensor-core GEMM tiles timed out waiting for their MMAs\n", st.timeout);
        if (st.drain_timeout)
            fprintf(stderr, "pastix_gpu: %d CTAs gave up waiting for their own TMA loads after a time-out: the "
                            "factorization's results are undefined\n", st.drain_timeout);
        C.fact_done = -1;
        return PASTIX_GPU_ERR_INTERNAL;
    }
    C.iparm[PGPU_IPARM_STATIC_PIVOTING] = st.nbpivots;
    const double fl = C.thflops[zc ? 1 : 0][fmode == FM_GETRF ? 1 : (fm_ldl(fmode) ? 2 : 0)];
    C.dparm[PGPU_DPARM_FACT_TIME] = ms * 1e-3;
    C.dparm[PGPU_DPARM_FACT_THFLOPS] = fl;
    C.dparm[PGPU_DPARM_FACT_FLOPS] = fl / (ms * 1e-3) / 1e9;
    C.coef_float = mixed;
    C.fact_done = fact;
    C.fact_mode = fmode;
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
// Solve on a permuted device RHS block W (factor precision, ld = n):
// sopalin/sequential_ztrsm.c:591 with the uplo/trans/diag choice of
// sopalin/pastix_task_solve.c:600-650 (forward L; for LDL the diagonal
// solve, sequential_zdiag.c; backward op(L)^t or U).
// --------------------------------------------------------------------------
// One launch of the dataflow solve over run `run`, forward or backward: a
// cooperative launch (every CTA resident), one CTA per SM.
template <typename T, int NR>
static int flow_launch(pastix_gpu_t &C, bool fwd, int run, const T *coefL, const T *inv, T *W, int ldb, bool ldl,
                       int cjp) {
    const int dir = fwd ? 0 : 1;
    auto kern = fwd ? k_solve_flow<T, NR, true> : k_solve_flow<T, NR, false>;
    const int vec_elems = (int)align16_elems<T>((size_t)std::max(C.flow_maxw, FLOW_MAXROWS) * NR);
    const size_t smem = (size_t)FLOW_S * FLOW_STAGE + (size_t)FLOW_S * vec_elems * sizeof(T);
    if ((size_t)vec_elems * sizeof(T) > (size_t)FLOW_VEC_BYTES) return PASTIX_GPU_ERR_INTERNAL;
    static size_t attr[2] = {0, 0};   // dynamic shared memory the kernel is set up for
    if (attr[dir] < smem) {
        PGPU_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr[dir] = smem;
    }
    int nsm = 0, per = 0;
    PGPU_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, C.device));
    PGPU_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, FLOW_THREADS, smem));
    if (per < 1) return PASTIX_GPU_ERR_INTERNAL;
    const unsigned long long nc = (unsigned long long)C.cblknbr;
    FlowArgs<T> a;
    a.m = C.meta;
    if (nsm != C.flow_G) return PASTIX_GPU_ERR_INTERNAL;   // (the schedule is for this many CTAs)
    a.tasks = C.d_flow_tasks[dir].p + C.flow_tptr[dir][run];
    a.ntasks = C.flow_tptr[dir][run + 1] - C.flow_tptr[dir][run];
    a.off = C.d_flow_off[dir].p + (size_t)run * 2 * (nsm + 1);
    a.epoch = ++C.flow_epoch[dir][run];
    a.fs = C.d_flow_state.p;
    unsigned long long *cnt = C.d_flow_cnt.p;
    const int *need = C.d_flow_need.p;
    a.k = FlowCounters{cnt, cnt + nc, cnt + 2 * nc, cnt + 3 * nc, cnt + 4 * nc,
                       need, need + nc, need + 2 * nc, need + 3 * nc};
    a.coef = coefL;
    a.inv = inv;
    a.B = W;
    a.Y = reinterpret_cast<T *>(C.d_flowY.p);
    a.Z = reinterpret_cast<T *>(C.d_flowZ.p);
    a.ldb = ldb;
    a.ldl = ldl ? 1 : 0;
    a.cjp = cjp;
    a.vec_elems = vec_elems;
    // PASTIX_GPU_SOLVE_PROFILE=3: per-task times, summarized per level on stderr (diagnostics)
    static const bool tprof = getenv("PASTIX_GPU_SOLVE_PROFILE") && getenv("PASTIX_GPU_SOLVE_PROFILE")[0] == '3';
    a.stamps = nullptr;
    if (tprof) {
        const size_t ns = 2 * (size_t)a.ntasks + (size_t)nsm * FRT_N;
        if (C.d_flow_stamps.n < ns) PGPU_CHECK(C.d_flow_stamps.alloc(ns));
        PGPU_CHECK(cudaMemsetAsync(C.d_flow_stamps.p, 0, ns * 8, C.stream));
        a.stamps = C.d_flow_stamps.p;
    }
    void *args[] = {&a};
    PGPU_CHECK(cudaLaunchCooperativeKernel((const void *)kern, dim3(nsm), dim3(FLOW_THREADS), args, smem, C.stream));
    C.flow_used = true;
    if (tprof) {
        // per level of the run: first start and last signal of its D / E tasks and of the O / G tasks of its
        // cblks, in microseconds from the first task's start
        std::vector<unsigned long long> t(2 * (size_t)a.ntasks + (size_t)nsm * FRT_N);
        std::vector<FlowTask> tk(a.ntasks);
        PGPU_CHECK(cudaMemcpyAsync(t.data(), a.stamps, t.size() * 8, cudaMemcpyDeviceToHost, C.stream));
        PGPU_CHECK(cudaMemcpyAsync(tk.data(), a.tasks, tk.size() * sizeof(FlowTask), cudaMemcpyDeviceToHost, C.stream));
        PGPU_CHECK(cudaStreamSynchronize(C.stream));
        unsigned long long t0 = ~0ull, t1 = 0;
        for (int i = 0; i < a.ntasks; i++) {
            t0 = std::min(t0, t[2 * i]);
            t1 = std::max(t1, t[2 * i + 1]);
        }
        const int la = C.flow_runs[run].x, lb = C.flow_runs[run].y;
        std::vector<double> lo(4 * (size_t)(lb - la), 1e30), hi(4 * (size_t)(lb - la), 0);
        for (int i = 0; i < a.ntasks; i++) {
            const int l = C.cblk_level[tk[i].c] - la, kd = (tk[i].hdr & 7) == FLOW_D ? 0 : 1;
            lo[4 * l + 2 * kd] = std::min(lo[4 * l + 2 * kd], (t[2 * i] - t0) * 1e-3);
            hi[4 * l + 2 * kd + 1] = std::max(hi[4 * l + 2 * kd + 1], (t[2 * i + 1] - t0) * 1e-3);
        }
        fprintf(stderr, "pastix_gpu dataflow %s levels %d..%d: %d tasks, %.1f us; per level (us): diag first..last, off first..last\n",
                fwd ? "forward" : "backward", la, lb - 1, a.ntasks, (t1 - t0) * 1e-3);
        for (int l = 0; l < lb - la; l++)
            fprintf(stderr, "  %d  %.1f..%.1f  %.1f..%.1f\n", la + l, lo[4 * l], hi[4 * l + 1], lo[4 * l + 2], hi[4 * l + 3]);
        double rt[FRT_N] = {0};
        for (int q = 0; q < nsm; q++)
            for (int j = 0; j < FRT_N; j++) rt[j] += t[2 * (size_t)a.ntasks + (size_t)q * FRT_N + j] / (double)nsm;
        fprintf(stderr, "  role waits, mean kcycles per CTA: fetch/empty %.1f fetch/ready %.1f vector/record %.1f "
                        "compute/full %.1f signal/done %.1f compute busy %.1f total %.1f\n",
                rt[FRT_F_EMPTY] * 1e-3, rt[FRT_F_READY] * 1e-3, rt[FRT_V_RECV] * 1e-3, rt[FRT_C_FULL] * 1e-3,
                rt[FRT_S_DONE] * 1e-3, rt[FRT_C_BUSY] * 1e-3, rt[FRT_TOTAL] * 1e-3);
    }
    return PASTIX_GPU_SUCCESS;
}

template <typename T>
static int flow_launch_nr(pastix_gpu_t &C, int nrhs, bool fwd, int run, const T *coefL, const T *inv, T *W,
                          int ldb, bool ldl, int cjp) {
    switch (nrhs) {
    case 1: return flow_launch<T, 1>(C, fwd, run, coefL, inv, W, ldb, ldl, cjp);
    case 2: return flow_launch<T, 2>(C, fwd, run, coefL, inv, W, ldb, ldl, cjp);
    case 4:
        if constexpr (sizeof(T) <= 8) return flow_launch<T, 4>(C, fwd, run, coefL, inv, W, ldb, ldl, cjp);
        return PASTIX_GPU_ERR_INTERNAL;
    default: return PASTIX_GPU_ERR_INTERNAL;
    }
}

// A wait of the dataflow solve that gave up (FlowState::err): the solve's
// results are undefined; its counters are cleared for the next one.
static int flow_check(pastix_gpu_t &C) {
    if (!C.flow_used) return PASTIX_GPU_SUCCESS;
    C.flow_used = false;
    FlowState fs;
    PGPU_CHECK(cudaMemcpy(&fs, C.d_flow_state.p, sizeof(fs), cudaMemcpyDeviceToHost));
    if (fs.err) {
        fprintf(stderr, "pastix_gpu: a wait of the dataflow solve timed out (%d)\n", fs.err);
        int rc = flow_reset(C);
        if (rc) return rc;
        PGPU_CHECK(cudaStreamSynchronize(C.stream));
        return PASTIX_GPU_ERR_INTERNAL;
    }
    return PASTIX_GPU_SUCCESS;
}

template <typename T>
// steps: PGPU_SOLVE_FORWARD | PGPU_SOLVE_DIAG | PGPU_SOLVE_BACKWARD (all three: a full solve)
static int solve_permuted(pastix_gpu_t &C, T *W, int nrhs, int *launches, int steps = 7) {
    const int fm = C.fact_mode;
    const bool lu = (fm == FM_GETRF), ldl = fm_ldl(fm);
    const int cjp = fm_conj(fm) ? 1 : 0;
    const T *coefL = reinterpret_cast<const T *>(C.d_coef.p);
    const T *coefU = lu ? coefL + C.coefnbr : coefL;
    cudaStream_t s = C.stream;
    const int ldb = C.n;
    int nl = 0;
    PGPU_CHECK(cudaFuncSetAttribute(k_fwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(k_bwd_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(k_fwd_off<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    PGPU_CHECK(cudaFuncSetAttribute(k_bwd_off<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT));
    // off-diagonal kernels: the chunk's rows (padded to 16 bytes) + the RHS values they need
    auto off_smem = [&](int mw, bool fwd) {
        const size_t wp = (size_t)round_up(mw, 16 / (int64_t)sizeof(T));
        const size_t rhs = fwd ? (size_t)nrhs * wp : (size_t)SOLVE_ROWS_PER_CHUNK * nrhs;
        return (align16_elems<T>(rhs) + (size_t)SOLVE_ROWS_PER_CHUNK * wp) * sizeof(T);
    };
    // PASTIX_GPU_SOLVE_PROFILE=1: device time per solve phase on stderr (diagnostics)
    static const bool prof = getenv("PASTIX_GPU_SOLVE_PROFILE") != nullptr;
    LaunchTimer tm(C);
    auto mark = [&](int k) { return prof ? tm.mark(k) : cudaSuccess; };
    // staged-panel rows of the diagonal kernels that fit next to the RHS block
    // and, on levels with diagonal-block inverses (panel TRSM done as a GEMM),
    // the rows of the inverse staged per chunk (ipch rows x w)
    static const bool inv_solve = !(getenv("PASTIX_GPU_SOLVE_INV") && std::strcmp(getenv("PASTIX_GPU_SOLVE_INV"), "0") == 0);
    const T *inv = (C.trsm_gemm && inv_solve) ? reinterpret_cast<const T *>(C.d_inv.p) : nullptr;
    auto diag_smem = [&](int l, int mw, int *pch, int *ipch) {
        const size_t es = sizeof(T);
        const size_t fixed = ((size_t)mw * nrhs + 32 * 33) * es;
        size_t dsm;
        *ipch = 0;
        if (inv && C.inv_ptr[l + 1] > C.inv_ptr[l]) {
            // rows of the inverse are staged padded to 16 bytes
            const size_t rowb = (size_t)round_up(mw, 16 / (int64_t)es) * es;
            const size_t fixed_i = ((size_t)2 * mw * nrhs + 16) * es;   // + alignment of the staged rows
            dsm = std::min<size_t>(SMEM_LIMIT, std::max(fixed_i + (size_t)128 * rowb, fixed + (size_t)mw * 33 * es));
            *ipch = dsm > fixed_i ? (int)std::min<size_t>(mw, (dsm - fixed_i) / rowb) : 0;
        } else {
            dsm = std::min<size_t>(SMEM_LIMIT, fixed + (size_t)std::max(mw, 1) * 33 * es);
        }
        *pch = dsm > fixed ? (int)std::min<size_t>(std::max(mw, 1), (dsm - fixed) / (33 * es)) : 0;
        return dsm;
    };
    // levels of narrow, short cblks: one warp per cblk, diagonal and off-diagonal parts in one launch
    auto small_level = [&](int l) { return C.lvl_maxw[l] <= 32 && C.lvl_maxh[l] <= SOLVE_SMALL_MAXH; };
    // runs of levels with diagonal-block inverses: one dataflow launch each way
    const bool flow = inv && C.tune[PGPU_TUNE_SOLVE_FLOW] != 0 &&
                      (nrhs == 1 || nrhs == 2 || (nrhs == 4 && sizeof(T) <= 8)) && nrhs <= FLOW_MAXRHS;
    auto flow_run_at = [&](int l, bool first) {
        if (flow)
            for (size_t r = 0; r < C.flow_runs.size(); r++)
                if ((first ? C.flow_runs[r].x : C.flow_runs[r].y - 1) == l) return (int)r;
        return -1;
    };
    for (int l = 0; l < ((steps & PGPU_SOLVE_FORWARD) ? C.nlevels : 0); l++) {
        const int ncb = C.lvl_ptr[l + 1] - C.lvl_ptr[l];
        tm.level = l;
        const int mw = C.lvl_maxw[l];
        const int run = flow_run_at(l, true);
        if (run >= 0) {
            PGPU_CHECK(mark(0));
            int rc = flow_launch_nr<T>(C, nrhs, true, run, coefL, inv, W, ldb, ldl, cjp);
            if (rc) return rc;
            nl++;
            l = C.flow_runs[run].y - 1;
            continue;
        }
        if (small_level(l)) {
            PGPU_CHECK(mark(0));
            const int *lc = C.d_lvl_cblks.p + C.lvl_ptr[l];
            const int un = (lu || ldl) ? 1 : 0;
            // right-hand sides 8 / 4 / 2 / 1 at a time in registers
            if (nrhs % 8 == 0) k_fwd_small<T, 8><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, W, ldb, nrhs, un);
            else if (nrhs % 4 == 0) k_fwd_small<T, 4><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, W, ldb, nrhs, un);
            else if (nrhs % 2 == 0) k_fwd_small<T, 2><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, W, ldb, nrhs, un);
            else k_fwd_small<T, 1><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, W, ldb, nrhs, un);
            nl++;
            continue;
        }
        int pch = 0;
        int ipch = 0;
        const size_t dsm = diag_smem(l, mw, &pch, &ipch);
        if (pch < std::min(32, mw) || (inv && C.inv_ptr[l + 1] > C.inv_ptr[l] && ipch < 1))
            return PASTIX_GPU_ERR_NOTIMPLEMENTED;
        PGPU_CHECK(mark(0));
        const int dthreads = (inv && C.inv_ptr[l + 1] > C.inv_ptr[l]) ? 1024 : 256;
        k_fwd_diag<T><<<ncb, dthreads, dsm, s>>>(
            C.meta, C.d_lvl_cblks.p + C.lvl_ptr[l], coefL, W, ldb, nrhs, (lu || ldl) ? 1 : 0, pch, inv,
            ldl ? 1 : 0, cjp, ipch);
        nl++;
        const int nch = C.solve_ptr[l + 1] - C.solve_ptr[l];
        if (nch) {
            PGPU_CHECK(mark(1));
            const size_t ysm = (size_t)round_up(mw, 16 / (int64_t)sizeof(T)) * nrhs * sizeof(T);
            const int2 *chp = C.d_solve_chunks.p + C.solve_ptr[l];
            if (nrhs == 1)
                k_fwd_off_direct<T, 1><<<nch, 256, ysm, s>>>(C.meta, chp, coefL, W, ldb, SOLVE_ROWS_PER_CHUNK);
            else if (nrhs == 2)
                k_fwd_off_direct<T, 2><<<nch, 256, ysm, s>>>(C.meta, chp, coefL, W, ldb, SOLVE_ROWS_PER_CHUNK);
            else if (nrhs == 4)
                k_fwd_off_direct<T, 4><<<nch, 256, ysm, s>>>(C.meta, chp, coefL, W, ldb, SOLVE_ROWS_PER_CHUNK);
            else if (nrhs == 8 && sizeof(T) <= 8)
                k_fwd_off_direct<T, 8><<<nch, 256, ysm, s>>>(C.meta, chp, coefL, W, ldb, SOLVE_ROWS_PER_CHUNK);
            else
                k_fwd_off<T><<<nch, 256, off_smem(mw, true), s>>>(C.meta, chp, coefL, W, ldb, nrhs,
                                                                  SOLVE_ROWS_PER_CHUNK);
            nl++;
        }
    }
    if (ldl && (steps & PGPU_SOLVE_DIAG)) {
        PGPU_CHECK(mark(2));
        k_diag_scale<T><<<std::min(C.cblknbr, 4096), 128, 0, s>>>(C.meta, coefL, W, ldb, nrhs);
        nl++;
    }
    for (int l = (steps & PGPU_SOLVE_BACKWARD) ? C.nlevels - 1 : -1; l >= 0; l--) {
        const int ncb = C.lvl_ptr[l + 1] - C.lvl_ptr[l];
        const int mw = C.lvl_maxw[l];
        tm.level = l;
        const int run = flow_run_at(l, false);
        if (run >= 0) {
            PGPU_CHECK(mark(4));
            int rc = flow_launch_nr<T>(C, nrhs, false, run, coefL, inv, W, ldb, ldl, lu ? 0 : cjp);
            if (rc) return rc;
            nl++;
            l = C.flow_runs[run].x;
            continue;
        }
        if (small_level(l)) {
            PGPU_CHECK(mark(4));
            const int *lc = C.d_lvl_cblks.p + C.lvl_ptr[l];
            const int up = lu ? 1 : 0, un = ldl ? 1 : 0, cj = lu ? 0 : cjp;
            if (nrhs % 8 == 0)
                k_bwd_small<T, 8><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, coefU, W, ldb, nrhs, up, un, cj);
            else if (nrhs % 4 == 0)
                k_bwd_small<T, 4><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, coefU, W, ldb, nrhs, up, un, cj);
            else if (nrhs % 2 == 0)
                k_bwd_small<T, 2><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, coefU, W, ldb, nrhs, up, un, cj);
            else
                k_bwd_small<T, 1><<<cdiv(ncb, 8), 256, 0, s>>>(C.meta, lc, ncb, coefL, coefU, W, ldb, nrhs, up, un, cj);
            nl++;
            continue;
        }
        const int nch = C.solve_ptr[l + 1] - C.solve_ptr[l];
        if (nch) {
            PGPU_CHECK(mark(3));
            const size_t xsm = (size_t)SOLVE_ROWS_PER_CHUNK * nrhs * sizeof(T);
            const int2 *chp = C.d_solve_chunks.p + C.solve_ptr[l];
            const int bcj = lu ? 0 : cjp;
            if (nrhs == 2)
                k_bwd_off_direct<T, 2><<<nch, 256, xsm, s>>>(C.meta, chp, coefU, W, ldb, SOLVE_ROWS_PER_CHUNK, bcj);
            else if (nrhs == 4)
                k_bwd_off_direct<T, 4><<<nch, 256, xsm, s>>>(C.meta, chp, coefU, W, ldb, SOLVE_ROWS_PER_CHUNK, bcj);
            else if (nrhs == 8)
                k_bwd_off_direct<T, 8><<<nch, 256, xsm, s>>>(C.meta, chp, coefU, W, ldb, SOLVE_ROWS_PER_CHUNK, bcj);
            else
                k_bwd_off<T><<<nch, 256, off_smem(mw, false), s>>>(C.meta, chp, coefU, W, ldb, nrhs,
                                                                   SOLVE_ROWS_PER_CHUNK, bcj);
            nl++;
        }
        int pch = 0;
        int ipch = 0;
        const size_t dsm = diag_smem(l, mw, &pch, &ipch);
        PGPU_CHECK(mark(4));
        const int dthreads = (inv && C.inv_ptr[l + 1] > C.inv_ptr[l]) ? 1024 : 256;
        k_bwd_diag<T><<<ncb, dthreads, dsm, s>>>(C.meta, C.d_lvl_cblks.p + C.lvl_ptr[l], coefL, W, ldb, nrhs,
                                            lu ? 1 : 0, ldl ? 1 : 0, lu ? 0 : cjp, pch, inv, ldl ? 1 : 0, ipch);
        nl++;
    }
    PGPU_CHECK(cudaGetLastError());
    if (prof) {
        PGPU_CHECK(mark(5));
        PGPU_CHECK(cudaStreamSynchronize(s));
        double ms[5];
        tm.collect(ms, 5);
        fprintf(stderr, "pastix_gpu solve profile (nrhs %d, %d levels): fwd_diag %.3f fwd_off %.3f diag %.3f "
                        "bwd_off %.3f bwd_diag %.3f ms\n", nrhs, C.nlevels, ms[0], ms[1], ms[2], ms[3], ms[4]);
        if (getenv("PASTIX_GPU_SOLVE_PROFILE")[0] == '2') {   // per level: fwd_diag fwd_off bwd_off bwd_diag
            std::vector<double> lv(5 * (size_t)C.nlevels, 0.0);
            for (int i = 0; i + 1 < tm.used; i++) {
                float t = 0;
                if (tm.kinds[i] >= 0 && tm.kinds[i] < 5 && tm.levels[i] >= 0 &&
                    cudaEventElapsedTime(&t, C.evpool[i], C.evpool[i + 1]) == cudaSuccess)
                    lv[5 * (size_t)tm.levels[i] + tm.kinds[i]] += t;
            }
            for (int l = 0; l < C.nlevels; l++)
                fprintf(stderr, "  level %d ncblk %d maxw %d: %.4f %.4f %.4f %.4f ms\n", l,
                        C.lvl_ptr[l + 1] - C.lvl_ptr[l], C.lvl_maxw[l], lv[5 * l + 0], lv[5 * l + 1], lv[5 * l + 3],
                        lv[5 * l + 4]);
        }
    }
    *launches += nl;
    return PASTIX_GPU_SUCCESS;
}

// bytes of one right-hand-side element (FP64 real or complex)
static size_t rhs_esz(const pastix_gpu_t &C) { return C.flttype == PGPU_COMPLEX64 ? 16 : 8; }
// bytes of one factor element
static size_t coef_esz(const pastix_gpu_t &C) { return (C.coef_float ? 4 : 8) * (C.flttype == PGPU_COMPLEX64 ? 2 : 1); }

static int ensure_work(pastix_gpu_t &C) {
    const size_t need = (size_t)C.n * SOLVE_MAXRHS * 16;
    if (C.d_work.n < need) {
        C.d_work.release();
        PGPU_CHECK(C.d_work.alloc(need));
    }
    if (C.d_rhs.n < (size_t)C.n * SOLVE_MAXRHS * 2) PGPU_CHECK(C.d_rhs.alloc((size_t)C.n * SOLVE_MAXRHS * 2));
    return PASTIX_GPU_SUCCESS;
}

// Permute in (down-casting for single-precision factors), solve, permute out.
// permuted: dB is already in the factorization's numbering (only the cast
// to and from the factor precision happens around the solve steps)
template <typename S, typename T>
static int solve_block_t(pastix_gpu_t &C, S *dB, int64_t ldb, int nrhs, T *W, int *launches, int steps = 7,
                         bool permuted = false) {
    // complex128 factors: at most 8 right-hand sides per pass (shared-memory staging of the solve kernels)
    if (sizeof(T) == 16 && nrhs > 8) {
        int rc = solve_block_t<S, T>(C, dB, ldb, 8, W, launches, steps, permuted);
        if (rc) return rc;
        return solve_block_t<S, T>(C, dB + 8 * ldb, ldb, nrhs - 8, W, launches, steps, permuted);
    }
    cudaStream_t s = C.stream;
    const int n = C.n;
    const int grid = std::min(4096, cdiv((int64_t)n * nrhs, 256));
    const int *perm = permuted ? nullptr : C.d_peritab.p;
    k_permute<S, T><<<grid, 256, 0, s>>>(n, nrhs, perm, dB, ldb, W, n, 0);
    int rc = solve_permuted<T>(C, W, nrhs, launches, steps);
    if (rc) return rc;
    k_permute<T, S><<<grid, 256, 0, s>>>(n, nrhs, perm, W, n, dB, ldb, 1);
    *launches += 2;
    PGPU_CHECK(cudaGetLastError());
    return PASTIX_GPU_SUCCESS;
}

// Solve in place on a device FP64 (real or complex) block, user order,
// ld = ldb elements, with W as the permuted work block.
static int solve_device_block(pastix_gpu_t &C, void *dB, int64_t ldb, int nrhs, void *W, int *launches) {
    if (C.flttype == PGPU_COMPLEX64) {
        if (C.coef_float) return solve_block_t<cdouble, cfloat>(C, (cdouble *)dB, ldb, nrhs, (cfloat *)W, launches);
        return solve_block_t<cdouble, cdouble>(C, (cdouble *)dB, ldb, nrhs, (cdouble *)W, launches);
    }
    if (C.coef_float) return solve_block_t<double, float>(C, (double *)dB, ldb, nrhs, (float *)W, launches);
    return solve_block_t<double, double>(C, (double *)dB, ldb, nrhs, (double *)W, launches);
}

// Solve steps on right-hand sides already in the factorization's numbering
// (pastix_gpu_solve_steps): FP64 data goes through the cast of
// solve_block_t, factor-precision data is solved in place in the work block.
template <typename T>
static int steps_native(pastix_gpu_t &C, int steps, int nr, char *db, int64_t dld, int *launches) {
    cudaStream_t s = C.stream;
    T *W = reinterpret_cast<T *>(C.d_work.p);
    PGPU_CHECK(cudaMemcpy2DAsync(W, (size_t)C.n * sizeof(T), db, dld * sizeof(T), (size_t)C.n * sizeof(T), nr,
                                 cudaMemcpyDeviceToDevice, s));
    const int step_rhs = sizeof(T) == 16 ? 8 : nr;   // (complex128 factors: 8 at a time, as solve_block_t)
    for (int r = 0; r < nr; r += step_rhs) {
        int rc = solve_permuted<T>(C, W + (int64_t)r * C.n, std::min(step_rhs, nr - r), launches, steps);
        if (rc) return rc;
    }
    PGPU_CHECK(cudaMemcpy2DAsync(db, dld * sizeof(T), W, (size_t)C.n * sizeof(T), (size_t)C.n * sizeof(T), nr,
                                 cudaMemcpyDeviceToDevice, s));
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_solve_steps(pastix_gpu_t *ctx, int steps, int64_t nrhs, void *B, int64_t ldb,
                                      int flttype) {
    if (!ctx || !B || nrhs <= 0 || ldb < ctx->n || steps <= 0 || steps > 7) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (C.fact_done < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    const bool zc = (C.flttype == PGPU_COMPLEX64);
    const bool fp64_data = flttype == (zc ? PGPU_COMPLEX64 : PGPU_DOUBLE);
    const bool native = C.coef_float && flttype == (zc ? PGPU_COMPLEX32 : PGPU_FLOAT);
    if (!fp64_data && !native) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(C.device));
    int rc = ensure_work(C);
    if (rc) return rc;
    cudaStream_t s = C.stream;
    const bool dev = is_device_ptr(B);
    int launches = 0;
    PGPU_CHECK(cudaEventRecord(C.ev[2], s));
    const size_t es = fp64_data ? rhs_esz(C) : coef_esz(C);
    for (int64_t r0 = 0; r0 < nrhs; r0 += SOLVE_MAXRHS) {
        const int nr = (int)std::min<int64_t>(SOLVE_MAXRHS, nrhs - r0);
        char *hb = reinterpret_cast<char *>(B) + r0 * ldb * es;
        char *db = hb;
        int64_t dld = ldb;
        if (!dev) {
            db = reinterpret_cast<char *>(C.d_rhs.p);
            dld = C.n;
            PGPU_CHECK(cudaMemcpy2DAsync(db, C.n * es, hb, ldb * es, C.n * es, nr, cudaMemcpyHostToDevice, s));
        }
        if (fp64_data) {
            if (zc)
                rc = C.coef_float ? solve_block_t<cdouble, cfloat>(C, (cdouble *)db, dld, nr, (cfloat *)C.d_work.p,
                                                                   &launches, steps, true)
                                  : solve_block_t<cdouble, cdouble>(C, (cdouble *)db, dld, nr,
                                                                    (cdouble *)C.d_work.p, &launches, steps, true);
            else
                rc = C.coef_float ? solve_block_t<double, float>(C, (double *)db, dld, nr, (float *)C.d_work.p,
                                                                 &launches, steps, true)
                                  : solve_block_t<double, double>(C, (double *)db, dld, nr, (double *)C.d_work.p,
                                                                  &launches, steps, true);
        } else {
            rc = zc ? steps_native<cfloat>(C, steps, nr, db, dld, &launches)
                    : steps_native<float>(C, steps, nr, db, dld, &launches);
        }
        if (rc) return rc;
        if (!dev) PGPU_CHECK(cudaMemcpy2DAsync(hb, ldb * es, db, C.n * es, C.n * es, nr, cudaMemcpyDeviceToHost, s));
    }
    PGPU_CHECK(cudaEventRecord(C.ev[3], s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[2], C.ev[3]));
    C.stats[1] = launches;
    C.stats[4] = ms;
    return flow_check(C);
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
    const size_t es = rhs_esz(C);
    for (int64_t r0 = 0; r0 < nrhs; r0 += SOLVE_MAXRHS) {
        const int nr = (int)std::min<int64_t>(SOLVE_MAXRHS, nrhs - r0);
        char *hb = reinterpret_cast<char *>(B) + r0 * ldb * es;
        void *db;
        int64_t dld;
        if (dev) {
            db = hb;
            dld = ldb;
        } else {
            db = C.d_rhs.p;
            dld = C.n;
            PGPU_CHECK(cudaMemcpy2DAsync(db, C.n * es, hb, ldb * es, C.n * es, nr, cudaMemcpyHostToDevice, s));
        }
        rc = solve_device_block(C, db, dld, nr, C.d_work.p, &launches);
        if (rc) return rc;
        if (!dev) PGPU_CHECK(cudaMemcpy2DAsync(hb, ldb * es, db, C.n * es, C.n * es, nr, cudaMemcpyDeviceToHost, s));
    }
    PGPU_CHECK(cudaEventRecord(C.ev[3], s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[2], C.ev[3]));
    C.stats[1] = launches;
    C.stats[4] = ms;
    C.dparm[PGPU_DPARM_SOLV_TIME] = ms * 1e-3;
    return flow_check(C);
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
    const size_t esz = coef_esz(C);
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
    int launches = 0;
    for (int64_t r0 = 0; r0 < nrhs; r0 += SOLVE_MAXRHS) {
        const int nr = (int)std::min<int64_t>(SOLVE_MAXRHS, nrhs - r0);
        char *db = reinterpret_cast<char *>(dB) + r0 * ldb * rhs_esz(C);
        rc = solve_device_block(C, db, ldb, nr, scratch, &launches);
        if (rc) return rc;
    }
    PGPU_CHECK(cudaGetLastError());
    PGPU_CHECK(cudaStreamSynchronize(s));
    return flow_check(C);
}

// --------------------------------------------------------------------------
// Refinement (refinement/z_refine_grad.c:49 z_grad_smp, preconditioned CG;
// refinement/z_refine_gmres.c:49 z_gmres_smp).  Vectors in the user
// numbering (the SpMV matrix is permuted, so vectors are permuted in and out
// of it).  S is the device scalar (double / cdouble), HS its host twin.
// --------------------------------------------------------------------------
template <typename S> struct HostScalar { typedef double type; };
template <> struct HostScalar<cdouble> { typedef std::complex<double> type; };
static inline double to_dev(double v) { return v; }
static inline cdouble to_dev(const std::complex<double> &v) { return cdouble(v.real(), v.imag()); }
static inline double to_host(double v) { return v; }
static inline std::complex<double> to_host(const cdouble &v) { return std::complex<double>(v.re, v.im); }

template <typename S>
struct VecOps {
    typedef typename HostScalar<S>::type HS;
    pastix_gpu_t &C;
    int launches = 0;
    S *partial() { return reinterpret_cast<S *>(C.d_partial.p); }
    S *scalar() { return reinterpret_cast<S *>(C.d_scalar.p); }
    // sum conj(x) y (bvec_zdotc); x . x when y == nullptr
    HS dot(const S *x, const S *y) {
        const int nb = 256;
        k_dot_partial<S><<<nb, RED_THREADS, 0, C.stream>>>(C.n, x, y, partial());
        k_dot_final<S><<<1, RED_THREADS, 0, C.stream>>>(nb, partial(), scalar(), 0);
        launches += 2;
        S v;
        cudaMemcpyAsync(&v, scalar(), sizeof(S), cudaMemcpyDeviceToHost, C.stream);
        cudaStreamSynchronize(C.stream);
        return to_host(v);
    }
    double norm(const S *x) { return std::sqrt(std::real(dot(x, nullptr))); }
    void axpy(HS a, const S *x, S *y) {
        k_axpy<S><<<1024, 256, 0, C.stream>>>(C.n, to_dev(a), x, y);
        launches++;
    }
    void xpby(const S *z, HS beta, S *p) {
        k_xpby<S><<<1024, 256, 0, C.stream>>>(C.n, z, to_dev(beta), p);
        launches++;
    }
    void copy(const S *x, S *y) { cudaMemcpyAsync(y, x, C.n * sizeof(S), cudaMemcpyDeviceToDevice, C.stream); }
    void scal(double a, S *x) {
        k_scal<S><<<1024, 256, 0, C.stream>>>(C.n, a, x);
        launches++;
    }
    // y = alpha A x + beta y in the user numbering, the CSR's own (x and y
    // are distinct vectors at every call)
    void spmv(double alpha, const S *x, double beta, S *y) {
        const int n = C.n;
        const S *val = reinterpret_cast<const S *>(C.d_csr_val.p);
        k_spmv<S><<<cdiv((int64_t)n * 32, 256), 256, 0, C.stream>>>(n, C.d_csr_ptr.p, C.d_csr_col.p, val, alpha, x,
                                                                     beta, y);
        launches++;
    }
    int spsv(S *z) { return solve_device_block(C, z, C.n, 1, C.d_work.p, &launches); }
    // per-system 2-norms of x (batch segments)
    void seg_norms(const S *x, std::vector<double> &out) {
        const int ns = (int)C.seg.size() - 1;
        k_seg_sumsq<S><<<std::min(ns, 4096), RED_THREADS, 0, C.stream>>>(ns, C.d_seg.p, x, C.d_segss.p);
        launches++;
        out.resize(ns);
        cudaMemcpyAsync(out.data(), C.d_segss.p, ns * sizeof(double), cudaMemcpyDeviceToHost, C.stream);
        cudaStreamSynchronize(C.stream);
        for (auto &v : out) v = std::sqrt(v);
    }
};

// Stopping measure of the refinement: ||r||/||b||, or with batch segments the
// largest per-system ||r_s||/||b_s|| (each system's own test).
template <typename S>
static double resid_measure(pastix_gpu_t &C, VecOps<S> &V, const S *r, double normr, double normb,
                            const std::vector<double> &segb) {
    if (C.seg.size() < 3) return normr / normb;
    std::vector<double> sr;
    V.seg_norms(r, sr);
    double m = 0;
    for (size_t i = 0; i < sr.size(); i++) m = std::max(m, sr[i] / (segb[i] > 0 ? segb[i] : 1.0));
    return m;
}

template <typename S>
static int refine_cg(pastix_gpu_t &C, VecOps<S> &V, const S *b, S *x, double eps, int itermax, int *iters,
                     double *resid) {
    typedef typename HostScalar<S>::type HS;
    S *r = reinterpret_cast<S *>(C.d_r.p), *z = reinterpret_cast<S *>(C.d_z.p);
    S *p = reinterpret_cast<S *>(C.d_p.p), *ap = reinterpret_cast<S *>(C.d_ap.p);
    double normb = V.norm(b);
    if (normb == 0.) normb = 1;
    const double normx = V.norm(x);
    std::vector<double> segb;
    if (C.seg.size() >= 3) V.seg_norms(b, segb);
    V.copy(b, r);
    if (normx > 0.) V.spmv(-1.0, x, 1.0, r);
    double normr = V.norm(r);
    double resid_b = resid_measure(C, V, r, normr, normb, segb);
    V.copy(r, z);
    int rc = V.spsv(z);
    if (rc) return rc;
    V.copy(z, p);
    int it = 0;
    while (resid_b > eps && it < itermax) {
        it++;
        V.spmv(1.0, p, 0.0, ap);
        HS beta = V.dot(r, z);
        HS alpha = V.dot(ap, p);
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
        resid_b = resid_measure(C, V, r, normr, normb, segb);
    }
    *iters = it;
    *resid = resid_b;
    return PASTIX_GPU_SUCCESS;
}

// Givens rotation that zeroes b under a (z_refine_gmres.c:257-272 for real
// data).  For complex data the unitary rotation [c s; -conj(s) c] with c real
// (LAPACK zlartg's convention): the reference's complex form takes a complex
// cosine and omits the conjugations, which is not unitary.
static inline void givens(double a, double b, double eps, double &c, double &s) {
    double t = std::sqrt(a * a + b * b);
    if (std::fabs(t) <= eps) t = eps;
    c = a / t;
    s = b / t;
}
static inline void givens(std::complex<double> a, std::complex<double> b, double eps, double &c,
                          std::complex<double> &s) {
    const double aa = std::abs(a), ab = std::abs(b);
    double t = std::sqrt(aa * aa + ab * ab);
    if (t <= eps) t = eps;
    if (aa == 0.0) {
        c = 0.0;
        s = (ab > 0.0) ? std::conj(b) / ab : std::complex<double>(1.0);
        return;
    }
    c = aa / t;
    s = (a / aa) * std::conj(b) / t;
}
static inline double conj_h(double v) { return v; }
static inline std::complex<double> conj_h(const std::complex<double> &v) { return std::conj(v); }

// --------------------------------------------------------------------------
// GMRES(im), right preconditioned (refinement/z_refine_gmres.c:49
// z_gmres_smp, Saad Alg. 9.5): V holds the Krylov basis, W = M^{-1} V so the
// solution update needs no extra solve; modified Gram-Schmidt with the
// projections h_{j,i} = <v_j, w> kept in device memory (one host round trip
// per inner iteration, for the Givens rotations on the small Hessenberg
// matrix).
// --------------------------------------------------------------------------
template <typename S>
static int refine_gmres(pastix_gpu_t &C, VecOps<S> &V, const S *b, S *x, double eps, int itermax, int im,
                        int *iters_out, double *resid_out) {
    typedef typename HostScalar<S>::type HS;
    const int64_t n = C.n;
    const int im1 = im + 1;
    const size_t comp = sizeof(S) / sizeof(double);
    if (C.d_gmV.n < (size_t)n * im1 * comp) {
        PGPU_CHECK(C.d_gmV.alloc((size_t)n * im1 * comp));
        PGPU_CHECK(C.d_gmW.alloc((size_t)n * im * comp));
    }
    if (C.d_gmh.n < (size_t)2 * im1 * comp) PGPU_CHECK(C.d_gmh.alloc((size_t)2 * im1 * comp));
    cudaStream_t s = C.stream;
    S *gV = reinterpret_cast<S *>(C.d_gmV.p), *gW = reinterpret_cast<S *>(C.d_gmW.p);
    S *dh = reinterpret_cast<S *>(C.d_gmh.p);
    S *part = V.partial();
    std::vector<HS> H((size_t)im * im1, HS(0.0)), sn(im, HS(0.0)), G(im1, HS(0.0));
    std::vector<double> cs(im, 0.0);
    std::vector<S> hcol(im1);
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
        V.scal(1.0 / resid, gV);
        std::fill(G.begin(), G.end(), HS(0.0));
        G[0] = HS(resid);
        int i = -1;
        bool inflag = true;
        while (inflag) {
            i++;
            S *vi = gV + (int64_t)i * n, *wi = gW + (int64_t)i * n, *vn = gV + (int64_t)(i + 1) * n;
            V.copy(vi, wi);
            int rc = V.spsv(wi);                       // w_i = M^{-1} v_i
            if (rc) return rc;
            V.spmv(1.0, wi, 0.0, vn);                  // v_{i+1} = A w_i
            for (int j = 0; j <= i; j++) {             // modified Gram-Schmidt
                k_dot_partial<S><<<256, RED_THREADS, 0, s>>>(n, gV + (int64_t)j * n, vn, part);
                k_dot_final<S><<<1, RED_THREADS, 0, s>>>(256, part, dh + j, 0);
                k_axpy_dev<S><<<1024, 256, 0, s>>>(n, dh + j, -1.0, gV + (int64_t)j * n, vn);
                V.launches += 3;
            }
            k_dot_partial<S><<<256, RED_THREADS, 0, s>>>(n, vn, nullptr, part);
            k_dot_final<S><<<1, RED_THREADS, 0, s>>>(256, part, dh + i + 1, 1);
            V.launches += 2;
            PGPU_CHECK(cudaMemcpyAsync(hcol.data(), dh, (i + 2) * sizeof(S), cudaMemcpyDeviceToHost, s));
            PGPU_CHECK(cudaStreamSynchronize(s));
            const double norm = std::real(to_host(hcol[i + 1]));
            if (norm > 1e-50) V.scal(1.0 / norm, vn);
            HS *Hi = H.data() + (size_t)i * im1;
            for (int j = 0; j <= i + 1; j++) Hi[j] = to_host(hcol[j]);
            for (int j = 0; j < i; j++) {              // previous Givens rotations
                const HS tmp = Hi[j];
                Hi[j] = cs[j] * tmp + sn[j] * Hi[j + 1];
                Hi[j + 1] = cs[j] * Hi[j + 1] - conj_h(sn[j]) * tmp;
            }
            givens(Hi[i], Hi[i + 1], eps, cs[i], sn[i]);
            G[i + 1] = -conj_h(sn[i]) * G[i];
            G[i] = cs[i] * G[i];
            Hi[i] = cs[i] * Hi[i] + sn[i] * Hi[i + 1];
            resid = std::abs(G[i + 1]);
            resid_b = resid / normb;
            iters++;
            if (i + 1 >= im || resid_b <= eps || iters >= itermax) inflag = false;
        }
        // y = H^{-1} g (upper triangular, size i+1), x += W y
        const int k = i + 1;
        for (int r = k - 1; r >= 0; r--) {
            HS sum = G[r];
            for (int j = r + 1; j < k; j++) sum -= H[(size_t)j * im1 + r] * G[j];
            G[r] = sum / H[(size_t)r * im1 + r];
        }
        for (int j = 0; j < k; j++) hcol[j] = to_dev(G[j]);
        PGPU_CHECK(cudaMemcpyAsync(dh, hcol.data(), k * sizeof(S), cudaMemcpyHostToDevice, s));
        k_gemv_acc<S><<<1024, 256, 0, s>>>(n, k, gW, n, dh, x);
        V.launches++;
        PGPU_CHECK(cudaStreamSynchronize(s));
        if (iters >= itermax) outflag = false;
    }
    *iters_out = iters;
    *resid_out = resid_b;
    return PASTIX_GPU_SUCCESS;
}

static int ensure_refine_vectors(pastix_gpu_t &C) {
    const size_t n2 = (size_t)C.n * 2 * MULTI_MAX;   // complex, up to MULTI_MAX columns
    if (C.d_r.n < n2) {
        PGPU_CHECK(C.d_r.alloc(n2));
        PGPU_CHECK(C.d_z.alloc(n2));
        PGPU_CHECK(C.d_p.alloc(n2));
        PGPU_CHECK(C.d_ap.alloc(n2));
        PGPU_CHECK(C.d_x.alloc(n2));
        PGPU_CHECK(C.d_gm.alloc(2 * n2));
    }
    if (C.d_rhs.n < n2) PGPU_CHECK(C.d_rhs.alloc(n2));
    if (C.d_partial.n < (size_t)2 * 256 * MULTI_MAX) PGPU_CHECK(C.d_partial.alloc((size_t)2 * 256 * MULTI_MAX));
    if (C.d_scalar.n < (size_t)4 * MULTI_MAX) PGPU_CHECK(C.d_scalar.alloc((size_t)4 * MULTI_MAX));
    return ensure_work(C);
}

// --------------------------------------------------------------------------
// Lockstep refinement of k <= MULTI_MAX right-hand sides: the reference
// refines one column after the other (refinement/pastix_task_refine.c:120-161);
// here the k columns share every SpMV and preconditioner solve (one
// multi-RHS supernodal solve instead of k single ones) while each keeps its
// own scalars, stopping test and iteration count -- a converged column is
// frozen (step 0) while the others go on.
// --------------------------------------------------------------------------
template <typename S>
struct BlockOps {
    typedef typename HostScalar<S>::type HS;
    pastix_gpu_t &C;
    int k;
    int launches = 0;
    S *partial() { return reinterpret_cast<S *>(C.d_partial.p); }
    S *scal() { return reinterpret_cast<S *>(C.d_scalar.p); }
    // per-column conj(x_c) . y_c (or ||x_c||^2), launched only
    void dot_dev(const S *x, const S *y, S *out, int do_sqrt) {
        const int nb = 256;
        k_dot_partial_multi<S><<<dim3(nb, k), RED_THREADS, 0, C.stream>>>(C.n, x, y, partial());
        k_dot_final_multi<S><<<k, RED_THREADS, 0, C.stream>>>(nb, partial(), out, do_sqrt);
        launches += 2;
    }
    void dot(const S *x, const S *y, std::vector<HS> &out) {
        dot_dev(x, y, scal(), 0);
        std::vector<S> h(k);
        cudaMemcpyAsync(h.data(), scal(), k * sizeof(S), cudaMemcpyDeviceToHost, C.stream);
        cudaStreamSynchronize(C.stream);
        out.resize(k);
        for (int c = 0; c < k; c++) out[c] = to_host(h[c]);
    }
    void norm(const S *x, std::vector<double> &out) {
        std::vector<HS> d;
        dot(x, nullptr, d);
        out.resize(k);
        for (int c = 0; c < k; c++) out[c] = std::sqrt(std::real(d[c]));
    }
    void axpy(const std::vector<HS> &a, const S *x, S *y) {
        Coefs<S> cf;
        for (int c = 0; c < MULTI_MAX; c++) cf.v[c] = to_dev(c < k ? a[c] : HS(0.0));
        k_axpy_multi<S><<<1024, 256, 0, C.stream>>>(C.n, k, cf, x, y);
        launches++;
    }
    void xpby(const S *z, const std::vector<HS> &beta, S *p) {
        Coefs<S> cf;
        for (int c = 0; c < MULTI_MAX; c++) cf.v[c] = to_dev(c < k ? beta[c] : HS(0.0));
        k_xpby_multi<S><<<1024, 256, 0, C.stream>>>(C.n, k, z, cf, p);
        launches++;
    }
    void scal(const std::vector<double> &a, S *x) {
        Coefs<double> cf;
        for (int c = 0; c < MULTI_MAX; c++) cf.v[c] = c < k ? a[c] : 1.0;
        k_scal_multi<S><<<1024, 256, 0, C.stream>>>(C.n, k, cf, x);
        launches++;
    }
    void copy(const S *x, S *y) {
        cudaMemcpyAsync(y, x, (size_t)C.n * k * sizeof(S), cudaMemcpyDeviceToDevice, C.stream);
    }
    // (the CSR is in the user numbering, as the vectors: no permutation; x
    // and y are distinct vectors at every call)
    void spmv(double alpha, const S *x, double beta, S *y) {
        const int n = C.n;
        const S *val = reinterpret_cast<const S *>(C.d_csr_val.p);
        if (C.csr_nnz <= (int64_t)16 * n)   // short rows: one thread per row
            k_spmv_rows_multi<S><<<std::min(cdiv(n, 256), 8 * 148), 256, 0, C.stream>>>(
                n, k, C.d_csr_ptr.p, C.d_csr_col.p, val, alpha, x, beta, y);
        else
            k_spmv_multi<S><<<cdiv((int64_t)n * 32, 256), 256, 0, C.stream>>>(n, k, C.d_csr_ptr.p, C.d_csr_col.p,
                                                                               val, alpha, x, beta, y);
        launches++;
    }
    int spsv(S *z) { return solve_device_block(C, z, C.n, k, C.d_work.p, &launches); }
    // per column: ||r_c|| / ||b_c||, or with batch segments the largest
    // per-system ratio of the column
    void measure(const S *r, const std::vector<double> &normr, const std::vector<double> &normb,
                 const std::vector<double> &segb, std::vector<double> &out) {
        out.resize(k);
        if (C.seg.size() < 3) {
            for (int c = 0; c < k; c++) out[c] = normr[c] / normb[c];
            return;
        }
        const int ns = (int)C.seg.size() - 1;
        std::vector<double> sr((size_t)ns * k);
        k_seg_sumsq_multi<S><<<dim3(std::min(ns, 4096), k), RED_THREADS, 0, C.stream>>>(ns, C.d_seg.p, C.n, r,
                                                                                      C.d_segss.p);
        launches++;
        cudaMemcpyAsync(sr.data(), C.d_segss.p, sr.size() * sizeof(double), cudaMemcpyDeviceToHost, C.stream);
        cudaStreamSynchronize(C.stream);
        for (int c = 0; c < k; c++) {
            double m = 0;
            for (int i = 0; i < ns; i++) {
                const double sb = segb[(size_t)c * ns + i];
                m = std::max(m, std::sqrt(sr[(size_t)c * ns + i]) / (sb > 0 ? sb : 1.0));
            }
            out[c] = m;
        }
    }
    void seg_norms(const S *x, std::vector<double> &out) {
        if (C.seg.size() < 3) return;
        const int ns = (int)C.seg.size() - 1;
        out.resize((size_t)ns * k);
        k_seg_sumsq_multi<S><<<dim3(std::min(ns, 4096), k), RED_THREADS, 0, C.stream>>>(ns, C.d_seg.p, C.n, x,
                                                                                      C.d_segss.p);
        launches++;
        cudaMemcpyAsync(out.data(), C.d_segss.p, out.size() * sizeof(double), cudaMemcpyDeviceToHost, C.stream);
        cudaStreamSynchronize(C.stream);
        for (auto &v : out) v = std::sqrt(v);
    }
};

// Preconditioned CG (refinement/z_refine_grad.c:49) on k columns in lockstep.
template <typename S>
static int refine_cg_block(pastix_gpu_t &C, BlockOps<S> &V, const S *b, S *x, double eps, int itermax,
                           std::vector<int> &iters, std::vector<double> &resid) {
    typedef typename HostScalar<S>::type HS;
    const int k = V.k;
    S *r = reinterpret_cast<S *>(C.d_r.p), *z = reinterpret_cast<S *>(C.d_z.p);
    S *p = reinterpret_cast<S *>(C.d_p.p), *ap = reinterpret_cast<S *>(C.d_ap.p);
    std::vector<double> normb, normx, normr, segb, res;
    V.norm(b, normb);
    for (auto &v : normb)
        if (v == 0.) v = 1;
    V.norm(x, normx);
    V.seg_norms(b, segb);
    V.copy(b, r);
    V.spmv(-1.0, x, 1.0, r);
    V.norm(r, normr);
    V.measure(r, normr, normb, segb, res);
    iters.assign(k, 0);
    std::vector<char> active(k);
    bool any = false;
    for (int c = 0; c < k; c++) any |= (active[c] = res[c] > eps && itermax > 0);
    if (any) {
        V.copy(r, z);
        int rc = V.spsv(z);
        if (rc) return rc;
        V.copy(z, p);
    }
    std::vector<HS> beta, alpha, alpha2, step(k), mstep(k);
    while (any) {
        V.spmv(1.0, p, 0.0, ap);
        V.dot(r, z, beta);
        V.dot(ap, p, alpha);
        for (int c = 0; c < k; c++) {
            step[c] = active[c] ? beta[c] / alpha[c] : HS(0.0);
            mstep[c] = -step[c];
        }
        V.axpy(step, p, x);
        V.axpy(mstep, ap, r);
        // the stopping test only reads r: it runs before the preconditioner
        // solve, which is skipped once every column has stopped (the
        // reference solves once more and discards z; x and r are the same)
        V.norm(r, normr);
        V.measure(r, normr, normb, segb, res);
        any = false;
        for (int c = 0; c < k; c++) {
            if (!active[c]) continue;
            iters[c]++;
            active[c] = res[c] > eps && iters[c] < itermax;
            any |= active[c];
        }
        if (!any) break;
        V.copy(r, z);
        int rc = V.spsv(z);
        if (rc) return rc;
        V.dot(r, z, alpha2);
        for (int c = 0; c < k; c++) beta[c] = active[c] ? alpha2[c] / beta[c] : HS(0.0);
        V.xpby(z, beta, p);
    }
    resid = res;
    return PASTIX_GPU_SUCCESS;
}

// GMRES(im), right preconditioned (refinement/z_refine_gmres.c:49), on k
// columns in lockstep: one Krylov basis per column (block j of V holds v_j
// of every column), per-column Hessenberg matrices and Givens rotations on
// the host.  A column leaves the inner loop when it converges or fills its
// basis; the restart cycle ends when every column has left it.
template <typename S>
static int refine_gmres_block(pastix_gpu_t &C, BlockOps<S> &V, const S *b, S *x, double eps, int itermax, int im,
                              std::vector<int> &iters_out, std::vector<double> &resid_out) {
    typedef typename HostScalar<S>::type HS;
    const int k = V.k;
    const int64_t n = C.n, nk = (int64_t)n * k;
    const int im1 = im + 1;
    const size_t comp = sizeof(S) / sizeof(double);
    if (C.d_gmV.n < (size_t)nk * im1 * comp) {
        PGPU_CHECK(C.d_gmV.alloc((size_t)nk * im1 * comp));
        PGPU_CHECK(C.d_gmW.alloc((size_t)nk * im * comp));
    }
    if (C.d_gmh.n < (size_t)2 * im1 * k * comp) PGPU_CHECK(C.d_gmh.alloc((size_t)2 * im1 * k * comp));
    cudaStream_t s = C.stream;
    S *gV = reinterpret_cast<S *>(C.d_gmV.p), *gW = reinterpret_cast<S *>(C.d_gmW.p);
    S *dh = reinterpret_cast<S *>(C.d_gmh.p);     // [j][c]
    std::vector<std::vector<HS>> H(k, std::vector<HS>((size_t)im * im1, HS(0.0))), G(k, std::vector<HS>(im1)),
        sn(k, std::vector<HS>(im));
    std::vector<std::vector<double>> cs(k, std::vector<double>(im, 0.0));
    std::vector<S> hcol((size_t)im1 * k);
    std::vector<double> normb, normx, rr, segb, resid(k, 0.0), resid_b(k, 0.0), scl(k);
    V.norm(b, normb);
    for (auto &v : normb)
        if (v == 0.) v = 1;
    V.norm(x, normx);
    V.seg_norms(b, segb);
    std::vector<int> iters(k, 0), kc(k, 0);
    std::vector<char> out(k, 1), in(k, 0), cyc(k, 0);
    while (true) {
        // r0 = b - A x for every column
        V.copy(b, gV);
        V.spmv(-1.0, x, 1.0, gV);
        V.norm(gV, rr);
        V.measure(gV, rr, normb, segb, resid_b);
        bool any = false;
        for (int c = 0; c < k; c++) {
            if (out[c] && resid_b[c] <= eps) out[c] = 0;
            cyc[c] = in[c] = out[c];
            any |= out[c];
            scl[c] = out[c] ? 1.0 / rr[c] : 1.0;
            if (out[c]) {
                std::fill(G[c].begin(), G[c].end(), HS(0.0));
                G[c][0] = HS(rr[c]);
            }
        }
        if (!any) break;
        V.scal(scl, gV);
        int i = -1;
        bool inner = true;
        while (inner) {
            i++;
            S *vi = gV + (int64_t)i * nk, *wi = gW + (int64_t)i * nk, *vn = gV + (int64_t)(i + 1) * nk;
            V.copy(vi, wi);
            int rc = V.spsv(wi);                      // w_i = M^{-1} v_i
            if (rc) return rc;
            V.spmv(1.0, wi, 0.0, vn);                 // v_{i+1} = A w_i
            for (int j = 0; j <= i; j++) {            // modified Gram-Schmidt, per column
                V.dot_dev(gV + (int64_t)j * nk, vn, dh + (size_t)j * k, 0);
                k_axpy_multi_dev<S><<<1024, 256, 0, s>>>(n, k, dh + (size_t)j * k, -1.0, gV + (int64_t)j * nk, vn);
                V.launches++;
            }
            V.dot_dev(vn, nullptr, dh + (size_t)(i + 1) * k, 1);
            PGPU_CHECK(cudaMemcpyAsync(hcol.data(), dh, (size_t)(i + 2) * k * sizeof(S), cudaMemcpyDeviceToHost, s));
            PGPU_CHECK(cudaStreamSynchronize(s));
            inner = false;
            for (int c = 0; c < k; c++) {
                const double nrm = std::real(to_host(hcol[(size_t)(i + 1) * k + c]));
                scl[c] = (in[c] && nrm > 1e-50) ? 1.0 / nrm : 1.0;
                if (!in[c]) continue;
                HS *Hi = H[c].data() + (size_t)i * im1;
                for (int j = 0; j <= i + 1; j++) Hi[j] = to_host(hcol[(size_t)j * k + c]);
                for (int j = 0; j < i; j++) {          // previous Givens rotations
                    const HS tmp = Hi[j];
                    Hi[j] = cs[c][j] * tmp + sn[c][j] * Hi[j + 1];
                    Hi[j + 1] = cs[c][j] * Hi[j + 1] - conj_h(sn[c][j]) * tmp;
                }
                givens(Hi[i], Hi[i + 1], eps, cs[c][i], sn[c][i]);
                G[c][i + 1] = -conj_h(sn[c][i]) * G[c][i];
                G[c][i] = cs[c][i] * G[c][i];
                Hi[i] = cs[c][i] * Hi[i] + sn[c][i] * Hi[i + 1];
                resid[c] = std::abs(G[c][i + 1]);
                resid_b[c] = resid[c] / normb[c];
                iters[c]++;
                kc[c] = i + 1;
                if (i + 1 >= im || resid_b[c] <= eps || iters[c] >= itermax) in[c] = 0;
                inner |= (bool)in[c];
            }
            V.scal(scl, vn);
        }
        // per column: y = H^{-1} g, x_c += W_c y
        for (int c = 0; c < k; c++) {
            if (!cyc[c]) continue;
            std::vector<HS> &Gc = G[c];
            const int kk = kc[c];
            for (int r = kk - 1; r >= 0; r--) {
                HS sum = Gc[r];
                for (int j = r + 1; j < kk; j++) sum -= H[c][(size_t)j * im1 + r] * Gc[j];
                Gc[r] = sum / H[c][(size_t)r * im1 + r];
            }
            for (int j = 0; j < kk; j++) hcol[j] = to_dev(Gc[j]);
            PGPU_CHECK(cudaMemcpyAsync(dh + (size_t)c * im1, hcol.data(), kk * sizeof(S), cudaMemcpyHostToDevice, s));
            k_gemv_acc<S><<<1024, 256, 0, s>>>(n, kk, gW + (int64_t)c * n, nk, dh + (size_t)c * im1,
                                               x + (int64_t)c * n);
            V.launches++;
            if (iters[c] >= itermax) out[c] = 0;
        }
        PGPU_CHECK(cudaStreamSynchronize(s));
    }
    iters_out = iters;
    resid_out = resid_b;
    return PASTIX_GPU_SUCCESS;
}

template <typename S>
static int refine_t(pastix_gpu_t &C, int64_t nrhs, const void *B, int64_t ldb, void *X, int64_t ldx, int *maxit,
                    double *maxres, int *launches) {
    cudaStream_t s = C.stream;
    double eps = C.dparm[PGPU_DPARM_EPSILON_REFINEMENT];
    if (eps < 0.) eps = 1e-12;   // refinement/pastix_task_refine.c:131-140 (double input)
    const int itermax = (int)C.iparm[PGPU_IPARM_ITERMAX];
    const int method = (int)C.iparm[PGPU_IPARM_REFINEMENT];
    const int im = std::max<int>(1, (int)C.iparm[PGPU_IPARM_GMRES_IM]);
    const bool bdev = is_device_ptr(B), xdev = is_device_ptr(X);
    const size_t es = sizeof(S);
    for (int64_t r0 = 0; r0 < nrhs; r0 += MULTI_MAX) {
        const int k = (int)std::min<int64_t>(MULTI_MAX, nrhs - r0);
        BlockOps<S> V{C, k};
        const S *bcol = reinterpret_cast<const S *>(B) + r0 * ldb;
        S *xcol = reinterpret_cast<S *>(X) + r0 * ldx;
        S *db = reinterpret_cast<S *>(C.d_rhs.p), *dx = reinterpret_cast<S *>(C.d_x.p);
        PGPU_CHECK(cudaMemcpy2DAsync(db, C.n * es, bcol, ldb * es, C.n * es, k,
                                     bdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        PGPU_CHECK(cudaMemcpy2DAsync(dx, C.n * es, xcol, ldx * es, C.n * es, k,
                                     xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        std::vector<int> it;
        std::vector<double> res;
        int rc = (method == PGPU_REFINE_CG) ? refine_cg_block<S>(C, V, db, dx, eps, itermax, it, res)
                                            : refine_gmres_block<S>(C, V, db, dx, eps, itermax, im, it, res);
        if (rc) return rc;
        PGPU_CHECK(cudaMemcpy2DAsync(xcol, ldx * es, dx, C.n * es, C.n * es, k,
                                     xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
        for (int c = 0; c < k; c++) {
            *maxit = std::max(*maxit, it[c]);
            *maxres = std::max(*maxres, res[c]);
        }
        *launches += V.launches;
    }
    return PASTIX_GPU_SUCCESS;
}

static int refine_impl(pastix_gpu_t &C, int64_t nrhs, const void *B, int64_t ldb, void *X, int64_t ldx) {
    int rc = ensure_refine_vectors(C);
    if (rc) return rc;
    const int method = (int)C.iparm[PGPU_IPARM_REFINEMENT];
    if (method != PGPU_REFINE_CG && method != PGPU_REFINE_GMRES) return PASTIX_GPU_ERR_NOTIMPLEMENTED;
    cudaStream_t s = C.stream;
    int maxit = 0, launches = 0;
    double maxres = 0;
    PGPU_CHECK(cudaEventRecord(C.ev[4], s));
    rc = (C.flttype == PGPU_COMPLEX64) ? refine_t<cdouble>(C, nrhs, B, ldb, X, ldx, &maxit, &maxres, &launches)
                                       : refine_t<double>(C, nrhs, B, ldb, X, ldx, &maxit, &maxres, &launches);
    if (rc) return rc;
    PGPU_CHECK(cudaEventRecord(C.ev[5], s));
    PGPU_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    PGPU_CHECK(cudaEventElapsedTime(&ms, C.ev[4], C.ev[5]));
    C.stats[2] = launches;
    C.stats[5] = ms;
    C.iparm[PGPU_IPARM_NBITER] = maxit;
    C.dparm[PGPU_DPARM_RELATIVE_ERROR] = maxres;
    C.dparm[PGPU_DPARM_REFINE_TIME] = ms * 1e-3;
    return flow_check(C);
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
    const size_t es = rhs_esz(C);
    if (bdev && xdev) {
        // X := B, solve in place, then refine -- all on the device
        PGPU_CHECK(cudaMemcpy2DAsync(X, ldx * es, B, ldb * es, C.n * es, nrhs, cudaMemcpyDeviceToDevice, C.stream));
        int rc = pastix_gpu_solve(ctx, nrhs, X, ldx);
        if (rc) return rc;
        return refine_impl(C, nrhs, B, ldb, X, ldx);
    }
    // host buffers: B crosses once, X comes back once
    const size_t words = (size_t)C.n * nrhs * (es / 8);
    if (C.d_sr_b.n < words) {
        PGPU_CHECK(C.d_sr_b.alloc(words));
        PGPU_CHECK(C.d_sr_x.alloc(words));
    }
    double *db = C.d_sr_b.p, *dx = C.d_sr_x.p;
    PGPU_CHECK(cudaMemcpy2DAsync(db, C.n * es, B, ldb * es, C.n * es, nrhs,
                                 bdev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, C.stream));
    PGPU_CHECK(cudaMemcpyAsync(dx, db, words * 8, cudaMemcpyDeviceToDevice, C.stream));
    int rc = pastix_gpu_solve(ctx, nrhs, dx, C.n);
    if (rc) return rc;
    rc = refine_impl(C, nrhs, db, C.n, dx, C.n);
    if (rc) return rc;
    PGPU_CHECK(cudaMemcpy2DAsync(X, ldx * es, dx, C.n * es, C.n * es, nrhs,
                                 xdev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, C.stream));
    PGPU_CHECK(cudaStreamSynchronize(C.stream));
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_set_segments(pastix_gpu_t *ctx, int64_t nseg, const int64_t *segptr) {
    if (!ctx || nseg < 0 || (nseg > 0 && !segptr)) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (nseg == 0) {
        C.seg.clear();
        return PASTIX_GPU_SUCCESS;
    }
    if (segptr[0] != 0 || segptr[nseg] != C.n) return PASTIX_GPU_ERR_BADPARAMETER;
    for (int64_t i = 0; i < nseg; i++)
        if (segptr[i + 1] < segptr[i]) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(C.device));
    C.seg.assign(segptr, segptr + nseg + 1);
    PGPU_CHECK(C.d_seg.upload(C.seg, C.stream));
    PGPU_CHECK(C.d_segss.alloc((size_t)nseg * MULTI_MAX));
    PGPU_CHECK(cudaStreamSynchronize(C.stream));
    return PASTIX_GPU_SUCCESS;
}

// --------------------------------------------------------------------------
// Learned cost model hooks: per-task timings recorded by the factorization
// itself, and a per-cblk cost that orders the work inside each level launch.
// --------------------------------------------------------------------------
extern "C" int pastix_gpu_record_tasks(pastix_gpu_t *ctx, int on) {
    if (!ctx) return PASTIX_GPU_ERR_BADPARAMETER;
    ctx->record = (on != 0);
    return PASTIX_GPU_SUCCESS;
}

static int task_records_impl(pastix_gpu_t *ctx, int64_t *count, int64_t *info, double *ns, int64_t *times);

extern "C" int pastix_gpu_task_records(pastix_gpu_t *ctx, int64_t *count, int64_t *info, double *ns) {
    if (!info || !ns) return task_records_impl(ctx, count, nullptr, nullptr, nullptr);
    return task_records_impl(ctx, count, info, ns, nullptr);
}

extern "C" int pastix_gpu_task_times(pastix_gpu_t *ctx, int64_t *count, int64_t *times) {
    if (!times) return task_records_impl(ctx, count, nullptr, nullptr, nullptr);
    std::vector<int64_t> info(8 * std::max<int64_t>(*count, 0));
    std::vector<double> ns(std::max<int64_t>(*count, 0));
    return task_records_impl(ctx, count, info.data(), ns.data(), times);
}

static int task_records_impl(pastix_gpu_t *ctx, int64_t *count, int64_t *info, double *ns, int64_t *times) {
    if (!ctx || !count) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    if (C.fact_done < 0 || !C.record || C.plan_fact < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    const int64_t cnt[4] = {C.cblknbr, (int64_t)C.h_trsm.size(), (int64_t)C.h_tiles.size(),
                            (int64_t)C.h_tctiles.size()};
    const int64_t total = cnt[0] + cnt[1] + cnt[2] + cnt[3];
    if (!info || !ns) {
        *count = total;
        return PASTIX_GPU_SUCCESS;
    }
    if (*count < total) return PASTIX_GPU_ERR_BADPARAMETER;
    PGPU_CHECK(cudaSetDevice(C.device));
    std::vector<int64_t> t[4];
    for (int k = 0; k < 4; k++) {
        t[k].resize(2 * cnt[k]);
        if (cnt[k]) PGPU_CHECK(cudaMemcpy(t[k].data(), C.d_prof[k].p, 2 * cnt[k] * sizeof(int64_t),
                                          cudaMemcpyDeviceToHost));
    }
    int64_t r = 0;
    auto put = [&](int kind, int64_t c, int64_t a, int64_t b, int64_t cc, int64_t d, const int64_t *tt) {
        int64_t *o = info + 8 * r;
        o[0] = kind; o[1] = c; o[2] = a; o[3] = b; o[4] = cc; o[5] = d; o[6] = C.plan_esz; o[7] = C.plan_fmode;
        ns[r] = (double)(tt[1] - tt[0]);
        if (times) {
            times[2 * r] = tt[0];
            times[2 * r + 1] = tt[1];
        }
        r++;
    };
    for (int q = 0; q < C.cblknbr; q++) {   // panel CTAs, in launch order (lvl_cblks)
        const int c = C.lvl_cblks[q];
        const int h = C.height[c], w = C.width[c];
        put(0, c, w, h, h <= C.plan_fuse ? h : w, C.fblok[c + 1] - C.fblok[c], &t[0][2 * q]);
    }
    for (int64_t i = 0; i < cnt[1]; i++) {
        const int4 ch = C.h_trsm[i];
        put(1, ch.x, C.width[ch.x], std::min(32, C.height[ch.x] - ch.y), ch.w, ch.z, &t[1][2 * i]);
    }
    for (int k = 2; k < 4; k++) {
        const auto &tl = (k == 2) ? C.h_tiles : C.h_tctiles;
        const int bm = (k == 2) ? GEMM_TM : TC_BM, bn = (k == 2) ? GEMM_TN : TC_BN;
        for (int64_t i = 0; i < cnt[k]; i++) {
            const GemmTask &g = C.h_tasks[tl[i].x];
            const int N = C.blrow[g.b] - C.bfrow[g.b] + 1;
            put(k, g.c, C.width[g.c], std::min(bm, g.M - tl[i].y * bm), std::min(bn, N - tl[i].z * bn), g.flags,
                &t[k][2 * i]);
        }
    }
    *count = total;
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_phase_log(pastix_gpu_t *ctx, int64_t *count, int64_t *info, double *times) {
    if (!ctx || !count) return PASTIX_GPU_ERR_BADPARAMETER;
    fact_marks_collect(*ctx);
    const int64_t n = (int64_t)ctx->phase_times.size() / 2;
    if (!info || !times) {
        *count = n;
        return PASTIX_GPU_SUCCESS;
    }
    const int64_t k = std::min<int64_t>(*count, n);
    std::memcpy(info, ctx->phase_info.data(), 3 * k * sizeof(int64_t));
    std::memcpy(times, ctx->phase_times.data(), 2 * k * sizeof(double));
    *count = k;
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_set_cblk_priority(pastix_gpu_t *ctx, const double *prio) {
    if (!ctx || ctx->cblknbr == 0) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    PGPU_CHECK(cudaSetDevice(C.device));
    for (int l = 0; l < C.nlevels; l++) {
        auto b = C.lvl_cblks.begin() + C.lvl_ptr[l], e = C.lvl_cblks.begin() + C.lvl_ptr[l + 1];
        if (prio)
            std::stable_sort(b, e, [prio](int x, int y) { return prio[x] > prio[y]; });
        else
            std::sort(b, e);
    }
    PGPU_CHECK(C.d_lvl_cblks.upload(C.lvl_cblks, C.stream));
    PGPU_CHECK(cudaStreamSynchronize(C.stream));
    C.plan_fact = -1;   // launch lists follow the new order
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_set_tuning(pastix_gpu_t *ctx, int key, int64_t value) {
    if (!ctx || key < 0 || key >= PGPU_TUNE_COUNT) return PASTIX_GPU_ERR_BADPARAMETER;
    if (key == PGPU_TUNE_MIXED_GEMM && (value < MG_FP32 || value > MG_3XF16)) return PASTIX_GPU_ERR_BADPARAMETER;
    if ((key == PGPU_TUNE_TRSM_GEMM_ROWS && value < 32) || (key == PGPU_TUNE_LA_RESERVED_SMS && value < 0) ||
        (key == PGPU_TUNE_TC_MIN_MN && value < 0) || (key == PGPU_TUNE_WIDE_PANEL && value < 0) || (key == PGPU_TUNE_TC_PAIR_MIN && value < -1) ||
        (key == PGPU_TUNE_GRAPH && (value < -1 || value > 1)))
        return PASTIX_GPU_ERR_BADPARAMETER;
    ctx->tune[key] = value;
    ctx->plan_fact = -1;   // the next numfact rebuilds its launch lists (and graph)
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_get_tuning(pastix_gpu_t *ctx, int key, int64_t *value) {
    if (!ctx || !value || key < 0 || key >= PGPU_TUNE_COUNT) return PASTIX_GPU_ERR_BADPARAMETER;
    *value = ctx->tune[key];
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

template <typename T>
static int coeftab_t(pastix_gpu_t &C, void *L, void *U, bool lu) {
    const size_t ncoef = (size_t)C.coefnbr * (lu ? 2 : 1);
    std::vector<T> h(ncoef);
    PGPU_CHECK(cudaMemcpy(h.data(), C.d_coef.p, ncoef * sizeof(T), cudaMemcpyDeviceToHost));
    host_relayout<T>(C, h, (T *)L, (T *)U, lu);
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_coeftab(pastix_gpu_t *ctx, void *L, void *U) {
    if (!ctx || ctx->fact_done < 0) return PASTIX_GPU_ERR_BADPARAMETER;
    auto &C = *ctx;
    PGPU_CHECK(cudaSetDevice(C.device));
    const bool lu = (C.fact_mode == FM_GETRF);
    if (C.flttype == PGPU_COMPLEX64)
        return C.coef_float ? coeftab_t<cfloat>(C, L, U, lu) : coeftab_t<cdouble>(C, L, U, lu);
    return C.coef_float ? coeftab_t<float>(C, L, U, lu) : coeftab_t<double>(C, L, U, lu);
}

extern "C" int pastix_gpu_stats(pastix_gpu_t *ctx, double *stats) {
    if (!ctx || !stats) return PASTIX_GPU_ERR_BADPARAMETER;
    fact_marks_collect(*ctx);
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
    for (auto &e : C->evpool2) cudaEventDestroy(e);
    for (auto &e : C->evpoolf) cudaEventDestroy(e);
    for (auto &e : C->la_events) cudaEventDestroy(e);
    if (C->fact_exec) cudaGraphExecDestroy(C->fact_exec);
    if (C->fact_graph) cudaGraphDestroy(C->fact_graph);
    if (C->stream2) {
        cudaStreamSynchronize(C->stream2);
        cudaStreamDestroy(C->stream2);
    }
    if (C->stream) cudaStreamDestroy(C->stream);
    delete C;   // every DArr member frees its device memory
    *pctx = nullptr;
}
