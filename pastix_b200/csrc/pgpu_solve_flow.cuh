// Dataflow solve of a run of levels whose cblks all hold the inverse of their
// diagonal block (kernels/solve_ztrsmsp.c:301 solve_cblk_ztrsmsp_forward and
// :450 solve_cblk_ztrsmsp_backward, the diagonal solve done as a product with
// the inverse, as the panel TRSM of these cblks was).
//
// Near the root of the elimination tree a level holds one to a few cblks, and
// one launch per level and phase pays a launch, a ramp and a drain for a few
// megabytes.  Here one launch per direction takes the whole run.  The run is
// cut into tasks of at most FLOW_MAXROWS rows in two lists, each in a
// dependency order: the critical tasks (the diagonal tasks, and the updates
// of the next level's cblks) and the others.  Task i of a list belongs to CTA
// i mod gridDim.x (the host stores each CTA's tasks of a list contiguously),
// and each task waits only for what it reads (per-cblk completion counters,
// no grid barrier):
//
//   forward   D(c, n0..)    y_c rows = s op(Binv_c rows) b_c       after every O(., c) of the run
//             O(c, f, r0..) b[rows] -= P_c rows y_c                after every D(c, .)
//   backward  G(c, f, r0..) b_c -= op(P_c rows)^t x[rows]         after x_f is final (f in the run)
//             E(c, n0..)    z_c += Binv_c rows^t (s b_c rows)      after every G(c, .)
//
// (s: d_n for LDL, op: conj for the Hermitian forms.)  Each CTA runs its tasks
// through a FLOW_S-stage pipeline of specialized warps, so that the fixed
// latencies of a task (its record, its dependency, its vector, its completion
// signal) overlap other tasks' work instead of adding up:
//   fetch warp   picks, of the CTA's next critical task and its next other
//                task, the one with the earlier deadline if its dependency is
//                met, else the other one if met (so neither list's head, when
//                it waits, holds up the other list), and puts the task record
//                (built on the host) into the stage and the factor rows it
//                reads -- contiguous, and independent of every other task --
//                into the stage's buffer by one bulk asynchronous copy;
//   vector warps (four, taking turns) load the vector part the task reads
//                (b_c, y_c or x at rows), many loads in flight per lane;
//   compute warps (eight) the products and their atomic updates;
//   signal warps (four, taking turns) publish the task's completion (fence,
//                counter), and the last diagonal task of a cblk moves its
//                solution into B (forward: from Y, where D tasks write y_c
//                while others still read b_c; backward: from Z, where the
//                partial sums meet, which is cleared again), then bx[c] = epoch.
//
// Both lists are sorted by one key that is a dependency order (a task waits
// only for tasks with smaller keys), every CTA is resident (cooperative
// launch) and takes the tasks of each list in order, so the unfinished task
// with the smallest key heads its list and has its inputs: the solve always
// progresses.  Counters grow by a fixed amount per launch of the
// run, so a launch waits for epoch x (tasks of the cblk) and no counter is
// reset between solves.  Every wait is bounded (about half a second for a
// dependency, two seconds for a stage); a wait that gives up sets
// FlowState::err, every role stops at its next task, and the host reports the
// solve as failed and clears the counters.
#pragma once

#include "pgpu_gemm_tma.cuh"
#include "pgpu_solve.cuh"

namespace pgpu {

constexpr int FLOW_S = 4;                 // pipeline stages per CTA
constexpr int FLOW_STAGE = 40 * 1024;     // bytes of one stage's factor rows
constexpr int FLOW_VEC_BYTES = 16 * 1024;   // bytes of one stage's vector part (at most)
constexpr int FLOW_MAXROWS = 32;          // rows of the factor per task
constexpr int FLOW_MAXRHS = 4;            // right-hand sides of one pass (1, 2 or 4; complex128: 1 or 2)
constexpr int FLOW_CWARPS = 8;            // compute warps
constexpr int FLOW_VWARPS = 4;            // vector warps (stage uses k with k mod 4 = the warp's index)
constexpr int FLOW_SWARPS = 4;            // signal warps (likewise)
constexpr int FLOW_W_FETCH = FLOW_CWARPS, FLOW_W_VEC = FLOW_CWARPS + 1, FLOW_W_SIG = FLOW_W_VEC + FLOW_VWARPS;
constexpr int FLOW_THREADS = 32 * (FLOW_W_SIG + FLOW_SWARPS);
constexpr long long FLOW_WAIT_CYCLES = 1000000000ll;

enum { FLOW_D = 0, FLOW_O = 1 };

// One task, built on the host: hdr = kind | flag << 3 | rows << 4 | deadline
// << 10 (flag: the target f is in the run -- forward O signals it, backward G
// waits for it; deadline: the list key of the task that needs this one);
// src: element offset of the task's factor rows from the inverse workspace
// (D / E) or from the coefficient array (O / G); aux: the panel rows'
// position in rowidx (O / G) or the cblk's coefficient offset (D / E); need:
// the per-launch value of the counter the task waits for (0: none).
struct __align__(16) FlowTask {
    int hdr, c, r0, f;
    int64_t src, aux;
    int w, ld, fc, need;
};
static_assert(sizeof(FlowTask) == 48, "three 16-byte vectors");

struct FlowState {
    int err, pad[3];
};

// Per-cblk counters (64-bit, monotone) and the per-launch increments they reach.
struct FlowCounters {
    unsigned long long *dd;    // forward: D tasks of c done
    unsigned long long *oin;   // forward: O tasks of the run into c done
    unsigned long long *go;    // backward: G tasks of c done
    unsigned long long *ed;    // backward: E tasks of c done
    unsigned long long *bx;    // backward: epoch once x_c is in B
    const int *nd, *noin, *ngo, *ned;
};

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(bytes) : "memory");
}


// Shared-memory loads by address in the shared window (the compute role reads
// its staged rows and vectors only through these, so that every one is an
// ld.shared and none a generic load)
__device__ __forceinline__ uint4 lds_u4(uint32_t a) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}
template <typename T> __device__ __forceinline__ T lds_t(uint32_t a);
template <> __device__ __forceinline__ float lds_t<float>(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ double lds_t<double>(uint32_t a) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ cfloat lds_t<cfloat>(uint32_t a) {
    float x, y;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "r"(a));
    return cfloat(x, y);
}
template <> __device__ __forceinline__ cdouble lds_t<cdouble>(uint32_t a) {
    double x, y;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "r"(a));
    return cdouble(x, y);
}

template <typename T> __device__ __forceinline__ T ldcg_v(const T *p) { return __ldcg(p); }
template <> __device__ __forceinline__ cfloat ldcg_v(const cfloat *p) {
    const float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
    return cfloat(v.x, v.y);
}
template <> __device__ __forceinline__ cdouble ldcg_v(const cdouble *p) {
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return cdouble(v.x, v.y);
}

template <typename T>
struct FlowArgs {
    Meta m;
    const FlowTask *tasks;   // the run's tasks; CTA q's: critical tasks[off[q] .. off[q + 1]) and
    const int *off;          // others tasks[off[G + 1 + q] .. off[G + 2 + q]), each in list order
    int ntasks;
    unsigned long long epoch;
    FlowState *fs;
    FlowCounters k;
    const T *coef;    // coefficient array (L, then U^t for LU): O / G rows, LDL diagonals
    const T *inv;     // diagonal-block inverses: D / E rows
    T *B, *Y, *Z;     // right-hand sides (ld ldb), forward y, backward partial sums
    int ldb;
    int ldl, cjp;     // LDL scaling; conj (forward: inverse and d; backward: the gathered panel)
    int vec_elems;    // elements of one stage's vector part
    unsigned long long *stamps;   // diagnostics (may be null): per task, global timer at compute start and at
                                  // signal; then per CTA FRT_N role times in clock cycles
};

// Diagnostics: per CTA, cycles the roles spent waiting (summed over a role's warps).
enum FlowRoleTime { FRT_F_EMPTY, FRT_F_READY, FRT_V_RECV, FRT_C_FULL, FRT_S_DONE, FRT_C_BUSY, FRT_TOTAL, FRT_N = 8 };

template <typename T, int NR, bool FWD>
__global__ void __launch_bounds__(FLOW_THREADS, 1) k_solve_flow(FlowArgs<T> a) {
    extern __shared__ __align__(128) unsigned char flow_smem[];
    __shared__ __align__(8) uint64_t full[FLOW_S], recv[FLOW_S], done[FLOW_S], empty[FLOW_S];
    __shared__ FlowTask rec[FLOW_S];
    __shared__ int rowsm[FLOW_S][FLOW_MAXROWS];   // O / G tasks: the panel rows' indices in B
    __shared__ int tix[FLOW_S];                    // the stage's task: index in the run's list (diagnostics)
    __shared__ int sfail;                          // this CTA saw a wait give up (mirrors FlowState::err)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int *err = &a.fs->err;
    const long long tstart = clock64();
    unsigned long long *roles = a.stamps ? a.stamps + 2 * (size_t)a.ntasks + (size_t)blockIdx.x * FRT_N : nullptr;
    auto role_add = [&](int slot, long long cyc) {
        if (roles && lane == 0) atomicAdd(roles + slot, (unsigned long long)cyc);
    };
    const unsigned long long ep = a.epoch;
    const int G = gridDim.x, q0 = blockIdx.x;
    const int hbeg = a.off[q0], nh_mine = a.off[q0 + 1] - hbeg;
    const int lbeg = a.off[G + 1 + q0], nl_mine = a.off[G + 2 + q0] - lbeg;
    const int nmine = nh_mine + nl_mine;
    // the counter a task waits for (with its per-launch value q.need)
    auto dep_of = [&](const FlowTask &q) -> const unsigned long long * {
        if (FWD) return (q.hdr & 7) == FLOW_D ? a.k.oin + q.c : a.k.dd + q.c;
        return (q.hdr & 7) == FLOW_D ? a.k.go + q.c : a.k.bx + q.f;
    };
    auto data = [&](int s) { return flow_smem + (size_t)s * FLOW_STAGE; };
    auto vec_of = [&](int s) {
        return reinterpret_cast<T *>(flow_smem + (size_t)FLOW_S * FLOW_STAGE) + (size_t)s * a.vec_elems;
    };
    // every role checks the CTA's flag per task (no global load on the fast path); the
    // fetch warp, when it waits for a dependency, also checks the grid's
    auto failed = [&]() { return *(volatile int *)&sfail != 0; };
    auto fail = [&](int code) {
        atomicExch(err, code);
        *(volatile int *)&sfail = 1;
    };
    if (tid == 0) {
        sfail = 0;
        for (int s = 0; s < FLOW_S; s++) {
            mbar_init(smem_u32(&full[s]), 32);   // the vector warp's lanes (+ the bulk copy's bytes)
            mbar_init(smem_u32(&recv[s]), 1);    // the fetch warp
            mbar_init(smem_u32(&done[s]), FLOW_CWARPS);
            mbar_init(smem_u32(&empty[s]), 1);   // the signal warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == FLOW_W_FETCH) {
        // ---- fetch: of the heads of the CTA's two lists, the one with the earlier deadline if its
        // dependency is met, else the other if met; its record and factor rows ----
        // (the lanes hold the next 32 records of each list, lane j: record base + j; lane 0 decides)
        const FlowTask *hl = a.tasks + hbeg, *ll = a.tasks + lbeg;
        int4 hr[3], lr[3];
        auto refill = [&](int4 (&r)[3], const FlowTask *list, int base, int n) {
            if (base + lane < n) {
                const int4 *p = reinterpret_cast<const int4 *>(list + base + lane);
                r[0] = __ldg(p);
                r[1] = __ldg(p + 1);
                r[2] = __ldg(p + 2);
            }
        };
        auto head = [&](const int4 (&r)[3], int j) {
            FlowTask q;
            int *o = reinterpret_cast<int *>(&q);
            const int *in = reinterpret_cast<const int *>(r);
#pragma unroll
            for (int e = 0; e < 12; e++) o[e] = __shfl_sync(0xffffffffu, in[e], j);
            return q;
        };
        const unsigned long long *known = nullptr;   // (lane 0) a counter seen at known_at: the CTA's
        unsigned long long known_at = 0;              // later tasks waiting for it need no load
        // (lane 0) the heads' counters, loaded as soon as a head changes so that the load's latency
        // passes while the fetch waits for a free stage; a value that meets the need is made an
        // acquire by the fence that follows it
        unsigned long long hval = 0, lval = 0;
        auto prefetch = [&](const FlowTask &q, unsigned long long &val) {
            if (lane == 0 && q.need) val = ld_relaxed_u64(dep_of(q));
        };
        auto ready = [&](const FlowTask &q, unsigned long long &val) -> bool {   // lane 0
            if (q.need == 0) return true;
            const unsigned long long *d = dep_of(q);
            const unsigned long long want = ep * (unsigned long long)q.need;
            if (d == known && known_at >= want) return true;
            if (val < want) val = ld_relaxed_u64(d);
            if (val >= want) {
                __threadfence();
                known = d;
                known_at = val;
                return true;
            }
            return false;
        };
        int kh = 0, kl = 0, k = 0;
        refill(hr, hl, 0, nh_mine);
        refill(lr, ll, 0, nl_mine);
        FlowTask hq = head(hr, 0), lq = head(lr, 0);
        if (nh_mine) prefetch(hq, hval);
        if (nl_mine) prefetch(lq, lval);
        for (; k < nmine; k++) {
            const int s = k % FLOW_S;
            int pick = -1;   // 0 critical, 1 other, -1 stop
            if (lane == 0) {
                const long long te = clock64();
                const bool got = !failed() &&
                                 (k < FLOW_S || mbar_wait(smem_u32(&empty[s]), (uint32_t)((k / FLOW_S - 1) & 1)));
                role_add(FRT_F_EMPTY, clock64() - te);
                if (got) {
                    const long long t0 = clock64();
                    const bool hfirst = kl >= nl_mine || (kh < nh_mine && (hq.hdr >> 10) <= (lq.hdr >> 10));
                    while (true) {
                        if (hfirst) {
                            if (kh < nh_mine && ready(hq, hval)) { pick = 0; break; }
                            if (kl < nl_mine && ready(lq, lval)) { pick = 1; break; }
                        } else {
                            if (kl < nl_mine && ready(lq, lval)) { pick = 1; break; }
                            if (kh < nh_mine && ready(hq, hval)) { pick = 0; break; }
                        }
                        if (*(volatile int *)err) {
                            *(volatile int *)&sfail = 1;
                            break;
                        }
                        if (clock64() - t0 > FLOW_WAIT_CYCLES) {
                            fail(1);
                            break;
                        }
                        __nanosleep(32);
                    }
                    role_add(FRT_F_READY, clock64() - t0);
                } else {
                    fail(1);
                }
                if (pick >= 0) {
                    const FlowTask q = pick == 0 ? hq : lq;
                    rec[s] = q;
                    tix[s] = pick == 0 ? hbeg + kh : lbeg + kl;
                    const uint32_t bytes = (uint32_t)(((q.hdr >> 4) & 63) * (size_t)q.ld * sizeof(T));
                    const T *src = ((q.hdr & 7) == FLOW_D ? a.inv : a.coef) + q.src;
                    mbar_expect_tx(smem_u32(&full[s]), bytes);
                    bulk_g2s(smem_u32(data(s)), src, bytes, smem_u32(&full[s]));
                    mbar_arrive(smem_u32(&recv[s]));
                }
            }
            pick = __shfl_sync(0xffffffffu, pick, 0);
            if (pick < 0) break;
            if (pick == 0) {
                if (++kh < nh_mine) {
                    if ((kh & 31) == 0) refill(hr, hl, kh, nh_mine);
                    hq = head(hr, kh & 31);
                    prefetch(hq, hval);
                }
            } else {
                if (++kl < nl_mine) {
                    if ((kl & 31) == 0) refill(lr, ll, kl, nl_mine);
                    lq = head(lr, kl & 31);
                    prefetch(lq, lval);
                }
            }
        }
        // copies still in flight (a later role stopped early) land before the CTA leaves
        if (lane == 0)
            for (int j = max(0, k - FLOW_S); j < k; j++)
                if (!mbar_wait(smem_u32(&full[j % FLOW_S]), (uint32_t)((j / FLOW_S) & 1))) fail(2);
    } else if (warp >= FLOW_W_VEC && warp < FLOW_W_VEC + FLOW_VWARPS) {
        // ---- vector: the vector part (GU loads in flight per lane) ----
        constexpr int GU = 8;
        T *vbase = nullptr;
        // v[e] = ld(e) for e < total
        auto gather = [&](int total, auto ld) {
            for (int b0 = 0; b0 < total; b0 += 32 * GU) {
                T tmp[GU];
#pragma unroll
                for (int u = 0; u < GU; u++) {
                    const int e = b0 + lane + 32 * u;
                    tmp[u] = e < total ? ld(e) : T(0);
                }
#pragma unroll
                for (int u = 0; u < GU; u++) {
                    const int e = b0 + lane + 32 * u;
                    if (e < total) vbase[e] = tmp[u];
                }
            }
        };
        for (int k = warp - FLOW_W_VEC; k < nmine; k += FLOW_VWARPS) {
            const int s = k % FLOW_S;
            const long long tw = clock64();
            const bool got = !failed() && mbar_wait(smem_u32(&recv[s]), (uint32_t)((k / FLOW_S) & 1));
            role_add(FRT_V_RECV, clock64() - tw);
            if (!got) {
                fail(1);
                break;
            }
            // (the fetch warp took the task once its dependency was met)
            const FlowTask q = rec[s];
            const int kind = q.hdr & 7, nr = (q.hdr >> 4) & 63;
            vbase = vec_of(s);
            const T *Bf = a.B + q.fc;
            if (FWD && kind == FLOW_D) {   // b_c, columns 0 .. r0 + nr - 1
                gather((q.r0 + nr) * NR, [&](int e) { return ldcg_v(Bf + (int64_t)(e % NR) * a.ldb + e / NR); });
            } else if (FWD) {              // y_c, and the rows the task updates
                const T *Yf = a.Y + q.fc;
                if (lane < nr) rowsm[s][lane] = __ldg(a.m.rowidx + q.aux + lane);
                gather(q.w * NR, [&](int e) { return ldcg_v(Yf + (int64_t)(e % NR) * a.ldb + e / NR); });
            } else if (kind == FLOW_O) {   // x at the task's rows
                if (lane < nr) rowsm[s][lane] = __ldg(a.m.rowidx + q.aux + lane);
                __syncwarp();
                const int *rw = rowsm[s];
                gather(nr * NR, [&](int e) { return ldcg_v(a.B + (int64_t)(e % NR) * a.ldb + rw[e / NR]); });
            } else {                       // v' = d t (LDL) or t, rows r0 ..
                gather(nr * NR, [&](int e) {
                    const int n = q.r0 + e / NR;
                    T x = ldcg_v(Bf + (int64_t)(e % NR) * a.ldb + n);
                    if (a.ldl) x = x * a.coef[q.aux + (int64_t)n * q.ld + n];
                    return x;
                });
            }
            mbar_arrive(smem_u32(&full[s]));
        }
    } else if (warp < FLOW_CWARPS) {
        // ---- compute ----
        for (int k = 0; k < nmine; k++) {
            const int s = k % FLOW_S;
            const long long tw = clock64();
            const bool got = !failed() && mbar_wait(smem_u32(&full[s]), (uint32_t)((k / FLOW_S) & 1));
            if (warp == 0) role_add(FRT_C_FULL, clock64() - tw);
            if (!got) {
                fail(1);
                break;
            }
            const FlowTask q = rec[s];
            const int kind = q.hdr & 7, nr = (q.hdr >> 4) & 63, w = q.w, ld = q.ld, fc = q.fc, r0 = q.r0;
            if (a.stamps && tid == 0) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                a.stamps[2 * (size_t)tix[s]] = t;
            }
            const uint32_t sP = smem_u32(data(s)), sv = smem_u32(vec_of(s));   // staged rows, vector part
            if (FWD) {
                // D  y_n = s op(Binv[n][k]) b_k, k <= n;  O  b[row_i] -= P[i][k] y_k.  Warp w takes rows
                // w, w + 8, .. (RW of them) together: lanes across k in 16-byte vectors, each vector of v
                // loaded once for all RW rows, every load of a pass independent of the others
                constexpr int VEC = 16 / sizeof(T), RW = FLOW_MAXROWS / FLOW_CWARPS;
                const bool dk = kind == FLOW_D;
                const int ilast = min(nr - 1, warp + FLOW_CWARPS * (RW - 1));
                const int kend = dk ? r0 + ilast + 1 : w;   // columns any of the warp's rows uses
                T acc[RW][NR];
#pragma unroll
                for (int u = 0; u < RW; u++)
#pragma unroll
                    for (int r = 0; r < NR; r++) acc[u][r] = T(0);
                if (warp < nr) {
                    for (int k0 = lane * VEC; k0 < kend; k0 += 32 * VEC) {
                        T vv[VEC][NR];
                        if (NR == 1 && k0 + VEC <= kend) {
                            T t4[VEC];
                            const uint4 u4 = lds_u4(sv + (uint32_t)k0 * sizeof(T));   // (16-byte aligned)
                            memcpy(t4, &u4, 16);
#pragma unroll
                            for (int q = 0; q < VEC; q++) vv[q][0] = t4[q];
                        } else {
#pragma unroll
                            for (int q = 0; q < VEC; q++)
#pragma unroll
                                for (int r = 0; r < NR; r++)
                                    vv[q][r] = k0 + q < kend ? lds_t<T>(sv + (uint32_t)((k0 + q) * NR + r) * sizeof(T))
                                                         : T(0);
                        }
                        T e[RW][VEC];
#pragma unroll
                        for (int u = 0; u < RW; u++) {
                            const int i = min(warp + FLOW_CWARPS * u, ilast);   // (rows past ilast: discarded)
                            const uint4 u4 = lds_u4(sP + (uint32_t)(i * ld + k0) * sizeof(T));
                            memcpy(e[u], &u4, 16);
                        }
#pragma unroll
                        for (int u = 0; u < RW; u++) {
                            const int klim = dk ? r0 + warp + FLOW_CWARPS * u + 1 : w;
#pragma unroll
                            for (int q = 0; q < VEC; q++) {
                                if (k0 + q < klim) {
                                    const T x = dk && a.cjp ? conj_v(e[u][q]) : e[u][q];
#pragma unroll
                                    for (int r = 0; r < NR; r++) acc[u][r] += x * vv[q][r];
                                }
                            }
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < RW; u++)
#pragma unroll
                    for (int r = 0; r < NR; r++)
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) acc[u][r] += shfl_xor_v(acc[u][r], o);
                // lane u stores row warp + 8 u
#pragma unroll
                for (int u = 0; u < RW; u++) {
                    const int i = warp + FLOW_CWARPS * u;
                    if (lane == u && i < nr) {
                        if (dk) {
                            const int n = r0 + i;
                            T d = T(1);
                            if (a.ldl) {
                                d = a.coef[q.aux + (int64_t)n * ld + n];
                                if (a.cjp) d = conj_v(d);
                            }
#pragma unroll
                            for (int r = 0; r < NR; r++)
                                a.Y[(int64_t)r * a.ldb + fc + n] = a.ldl ? acc[u][r] * d : acc[u][r];
                        } else {
                            const int grow = rowsm[s][i];
#pragma unroll
                            for (int r = 0; r < NR; r++) atomic_sub(&a.B[(int64_t)r * a.ldb + grow], acc[u][r]);
                        }
                    }
                }
            } else {
                // one thread per column: G  b_c[j] -= sum_i op(P[i][j]) x_i;  E  z_c[j] += sum_{n >= j} Binv[n][j] v'_n
                const int jend = kind == FLOW_O ? w : r0 + nr;
                for (int j = tid; j < jend; j += 32 * FLOW_CWARPS) {
                    T sm[NR];
#pragma unroll
                    for (int r = 0; r < NR; r++) sm[r] = T(0);
                    const int i0 = kind == FLOW_O ? 0 : max(0, j - r0);
#pragma unroll 8
                    for (int i = i0; i < nr; i++) {
                        T e = lds_t<T>(sP + (uint32_t)(i * ld + j) * sizeof(T));
                        if (kind == FLOW_O && a.cjp) e = conj_v(e);
#pragma unroll
                        for (int r = 0; r < NR; r++) sm[r] += e * lds_t<T>(sv + (uint32_t)(i * NR + r) * sizeof(T));
                    }
                    if (kind == FLOW_O) {
#pragma unroll
                        for (int r = 0; r < NR; r++) atomic_sub(&a.B[(int64_t)r * a.ldb + fc + j], sm[r]);
                    } else {
#pragma unroll
                        for (int r = 0; r < NR; r++) atomic_add(&a.Z[(int64_t)r * a.ldb + fc + j], sm[r]);
                    }
                }
            }
            __syncwarp();
            if (warp == 0) role_add(FRT_C_BUSY, clock64() - tw);
            if (lane == 0) mbar_arrive(smem_u32(&done[s]));
        }
    } else if (warp >= FLOW_W_SIG && warp < FLOW_W_SIG + FLOW_SWARPS) {
        // ---- signal: completion, and the cblk's solution into B after its last diagonal task ----
        for (int k = warp - FLOW_W_SIG; k < nmine; k += FLOW_SWARPS) {
            const int s = k % FLOW_S;
            const long long tw = clock64();
            const bool got = !failed() && mbar_wait(smem_u32(&done[s]), (uint32_t)((k / FLOW_S) & 1));
            role_add(FRT_S_DONE, clock64() - tw);
            if (!got) {
                fail(1);
                break;
            }
            const FlowTask q = rec[s];
            const int kind = q.hdr & 7, flag = (q.hdr >> 3) & 1, c = q.c;
            int last = 0;
            if (lane == 0) {
                __threadfence();   // the compute warps' stores and atomics of the task, before its counter
                if (FWD && kind == FLOW_D) {
                    last = atomicAdd(&a.k.dd[c], 1ull) + 1 == ep * (unsigned long long)a.k.nd[c];
                } else if (FWD) {
                    if (flag) atomicAdd(&a.k.oin[q.f], 1ull);
                } else if (kind == FLOW_O) {
                    atomicAdd(&a.k.go[c], 1ull);
                } else {
                    last = atomicAdd(&a.k.ed[c], 1ull) + 1 == ep * (unsigned long long)a.k.ned[c];
                }
                if (last) __threadfence();
            }
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                for (int e = lane; e < q.w * NR; e += 32) {
                    const int j = e / NR, r = e - j * NR;
                    const int64_t o = (int64_t)r * a.ldb + q.fc + j;
                    if (FWD) {
                        a.B[o] = ldcg_v(a.Y + o);
                    } else {
                        a.B[o] = ldcg_v(a.Z + o);
                        a.Z[o] = T(0);
                    }
                }
                __syncwarp();
                if (!FWD && lane == 0) {
                    __threadfence();
                    atomicExch(&a.k.bx[c], ep);
                }
            }
            __syncwarp();
            if (a.stamps && lane == 0) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                a.stamps[2 * (size_t)tix[s] + 1] = t;
            }
            if (lane == 0) mbar_arrive(smem_u32(&empty[s]));
        }
    }
    if (warp == 0) role_add(FRT_TOTAL, clock64() - tstart);
}

}  // namespace pgpu
