/*
 * pastix_gpu.h -- C ABI of the B200 numerical factorization and solve.
 *
 * This library replaces the numerical part of PaStiX ("sopalin") on one
 * NVIDIA B200: the coeftab lives in device memory and the diagonal-block
 * factorizations, panel TRSMs, update GEMMs with their indexed scatter-add,
 * the forward/backward solves and the iterative refinement run as CUDA
 * kernels.  Ordering, symbolic factorization and blend analysis stay on the
 * host: their output (the SolverMatrix cblk/blok/browtab arrays and the
 * ordering) is handed over once through pastix_gpu_structure().
 *
 * Every entry point takes plain pointers and sizes.  Integer tables are
 * int64_t (PaStiX built with PASTIX_INT64, its default); numerical arrays are
 * double / double _Complex as the reference's PastixDouble / PastixComplex64
 * data.  Return values are the reference's pastix_error_t codes
 * (include/pastix/api.h:368-376).
 *
 * The one reference-side plug point per entry point is named in its comment.
 */
#ifndef PASTIX_GPU_H
#define PASTIX_GPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PASTIX_GPU_API __attribute__((visibility("default")))
#else
#define PASTIX_GPU_API
#endif

/* pastix_error_t (include/pastix/api.h:368-376) */
#define PASTIX_GPU_SUCCESS          0
#define PASTIX_GPU_ERR_ALLOC        2
#define PASTIX_GPU_ERR_NOTIMPLEMENTED 3
#define PASTIX_GPU_ERR_OUTOFMEMORY  4
#define PASTIX_GPU_ERR_INTERNAL     6
#define PASTIX_GPU_ERR_BADPARAMETER 7

/* iparm / dparm indices used here, same values as include/pastix/api.h:35-186 */
#define PGPU_IPARM_VERBOSE          0
#define PGPU_IPARM_NNZEROS          2
#define PGPU_IPARM_FACTORIZATION   43
#define PGPU_IPARM_STATIC_PIVOTING 45
#define PGPU_IPARM_REFINEMENT      51
#define PGPU_IPARM_NBITER          52
#define PGPU_IPARM_ITERMAX         53
#define PGPU_IPARM_GMRES_IM        54
#define PGPU_IPARM_MIXED           71
#define PGPU_IPARM_SIZE            80
#define PGPU_DPARM_EPSILON_REFINEMENT 1
#define PGPU_DPARM_RELATIVE_ERROR     2
#define PGPU_DPARM_EPSILON_MAGN_CTRL  3
#define PGPU_DPARM_FACT_TIME         10
#define PGPU_DPARM_FACT_FLOPS        11
#define PGPU_DPARM_FACT_THFLOPS      12
#define PGPU_DPARM_SOLV_TIME         17
#define PGPU_DPARM_REFINE_TIME       22
#define PGPU_DPARM_A_NORM            23
#define PGPU_DPARM_SIZE              26

/* pastix_factotype_t (include/pastix/api.h:313-324) */
#define PGPU_FACT_POTRF 0
#define PGPU_FACT_SYTRF 1
#define PGPU_FACT_GETRF 2
#define PGPU_FACT_HETRF 4
/* spm_mtxtype_t values (PastixGeneral/Symmetric/Hermitian) */
#define PGPU_GENERAL   111
#define PGPU_SYMMETRIC 112
#define PGPU_HERMITIAN 113
/* spm_coeftype_t / pastix_coeftype_t values (input matrix: DOUBLE or
 * COMPLEX64; right-hand sides in the factor precision: FLOAT or COMPLEX32) */
#define PGPU_FLOAT     2
#define PGPU_DOUBLE    3
#define PGPU_COMPLEX32 4
#define PGPU_COMPLEX64 5
/* pastix_refine_t (include/pastix/api.h:273-278) */
#define PGPU_REFINE_GMRES 0
#define PGPU_REFINE_CG    1

typedef struct pastix_gpu_s pastix_gpu_t;

/*
 * Create a context on CUDA device `device`, copying the caller's iparm/dparm
 * arrays (IPARM_SIZE / DPARM_SIZE entries in the reference's order; NULL
 * keeps the reference defaults of common/api.c:411-560).
 * Replaces the GPU side of pastixInit (common/api.c:891).
 */
PASTIX_GPU_API int pastix_gpu_init( pastix_gpu_t **ctx, int device,
                     const int64_t *iparm, const double *dparm );

/*
 * Hand over the analysis result: the SolverMatrix of blend/solver.h:137-273
 * produced by pastix_subtask_blend (blend/pastix_subtask_blend.c:121).
 *   cblktab : (cblknbr+1) x 4  {fcolnum, lcolnum, first blok index, brownum}
 *   bloktab : bloknbr x 4      {frownum, lrownum, lcblknm, fcblknm}
 *   browtab : brownbr          (blend/solver.h:222)
 *   permtab, peritab : n       (pastix_order_t, include/pastix/order.h)
 * All indices 0-based.  The device coeftab is laid out and allocated here
 * (plug point: coeftabInit, sopalin/coeftab.c:204).
 */
PASTIX_GPU_API int pastix_gpu_structure( pastix_gpu_t *ctx, int64_t n,
                          int64_t cblknbr, const int64_t *cblktab,
                          int64_t bloknbr, const int64_t *bloktab,
                          int64_t brownbr, const int64_t *browtab,
                          const int64_t *permtab, const int64_t *peritab );

/*
 * Hand over the pattern of the user's matrix (0-based CSC; Symmetric and
 * Hermitian matrices give one triangle).  Builds the device-side bcsc
 * equivalents on the device: the fill-in map into the coeftab and the
 * full matrix in CSR (user numbering) the refinement multiplies by (its device time is
 * stats[15] of pastix_gpu_stats).  Replaces pastix_subtask_spm2bcsc
 * (sopalin/pastix_task_sopalin.c:93) / bcscInit (bcsc/bcsc.c:1887).
 */
PASTIX_GPU_API int pastix_gpu_spm( pastix_gpu_t *ctx, int mtxtype, int flttype, int64_t n,
                    const int64_t *colptr, const int64_t *rowptr );

/*
 * Numerical factorization of the matrix whose values (in the order of the
 * pattern given to pastix_gpu_spm) are at `values` -- host or device memory.
 * iparm[IPARM_FACTORIZATION] selects POTRF / GETRF / HETRF, and
 * iparm[IPARM_MIXED] = 1 factorizes in single precision.  Copies the values
 * in, scatters them into the coeftab and factorizes it.
 * Replaces pastix_task_numfact (sopalin/pastix_task_sopalin.c:637), i.e. the
 * bcsc2ctab and sopalin subtasks (plug point: sopalinFacto,
 * sopalin/pastix_task_sopalin.c:51-58).
 */
PASTIX_GPU_API int pastix_gpu_numfact( pastix_gpu_t *ctx, const void *values );

/*
 * Solve A X = B in place for `nrhs` right-hand sides (column-major, leading
 * dimension ldb, host or device memory).  Replaces pastix_task_solve
 * (sopalin/pastix_task_solve.c:753; plug point: ztrsm_table,
 * sopalin/sequential_ztrsm.c:536-552).
 */
PASTIX_GPU_API int pastix_gpu_solve( pastix_gpu_t *ctx, int64_t nrhs, void *B, int64_t ldb );

/*
 * Solve steps on right-hand sides already permuted into the factorization's
 * numbering (the pastix_rhs_t Bp of pastix_subtask_solve_adv,
 * sopalin/pastix_task_solve.c:511): steps is a mask of
 *   PGPU_SOLVE_FORWARD  the lower sweep, L y = b (unit L for LU and LDL),
 *   PGPU_SOLVE_DIAG     the diagonal step of LDL^t / LDL^h (z = D^-1 y),
 *   PGPU_SOLVE_BACKWARD the upper sweep (L^t / L^h x = z, or U x = y for LU).
 * Each step replaces one call through the reference's solve tables:
 * ztrsm_table (sopalin/sequential_ztrsm.c:536-552) for the sweeps and
 * zdiag_table (sopalin/sequential_zdiag.c:298) for the diagonal.  B holds
 * nrhs columns of leading dimension ldb in host or device memory; flttype is
 * the arithmetic of B: PGPU_DOUBLE / PGPU_COMPLEX64 (cast to the factor
 * precision and back on the device), or, for single-precision factors,
 * PGPU_FLOAT / PGPU_COMPLEX32 (the reference's mixed solve hands the sweeps
 * a single-precision copy of the right-hand sides).
 */
#define PGPU_SOLVE_FORWARD  1
#define PGPU_SOLVE_DIAG     2
#define PGPU_SOLVE_BACKWARD 4
PASTIX_GPU_API int pastix_gpu_solve_steps( pastix_gpu_t *ctx, int steps, int64_t nrhs, void *B, int64_t ldb,
                                           int flttype );

/*
 * Allocation-free solve: A X = B in place for `nrhs` right-hand sides that
 * already live in device memory (dB, column-major, leading dimension ldb),
 * using the factors of the last pastix_gpu_numfact.  No counterpart in the
 * reference: it exists for callers that cannot let a library allocate device
 * memory in the middle of their work -- applications whose own pool
 * allocator has already reserved the GPU's memory, and solve loops that must
 * not be stalled by cudaMalloc/cudaFree, which can synchronize the device.
 *
 * The call allocates nothing.  Its scratch (the permuted right-hand sides in
 * factor precision) is a fixed array of PASTIX_GPU_NOALLOC_SCRATCH_BYTES
 * (16 MiB) in the library's device memory, which every GPU that loads the
 * library holds until the process exits.  It holds up to 16 right-hand sides
 * at a time, so n * min(nrhs, 16) * (8 for FP64 factors, 4 for FP32) must not
 * exceed 16 MiB (e.g. n <= 131072 for 16 FP64 right-hand sides, n <= 2097152
 * for one); larger requests return PASTIX_GPU_ERR_BADPARAMETER without doing
 * any work.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, once per device); make that first call before any
 * stream capture.  All calls share the one array and it keeps the contents of
 * the last call (nothing needs clearing: every element used is written first),
 * so calls that overlap on the GPU -- from two contexts, threads or streams on
 * the same device -- race and must be serialized by the caller.  The address
 * is kept for the life of the process: a reset of the device (cudaDeviceReset,
 * or the primary context released and created again) invalidates it, so no
 * call may follow such a reset.
 * Returns when the solution is in dB.
 */
#define PASTIX_GPU_NOALLOC_SCRATCH_BYTES ( (size_t)16 << 20 )
PASTIX_GPU_API int pastix_gpu_solve_noalloc( pastix_gpu_t *ctx, int64_t nrhs, void *dB, int64_t ldb );

/*
 * Iterative refinement of X for A X = B (CG or GMRES, per
 * iparm[IPARM_REFINEMENT]; FP64 residuals, preconditioned by the factors)
 * to dparm[DPARM_EPSILON_REFINEMENT].  Replaces pastix_task_refine
 * (refinement/pastix_task_refine.c:231).
 */
PASTIX_GPU_API int pastix_gpu_refine( pastix_gpu_t *ctx, int64_t nrhs, const void *B, int64_t ldb,
                       void *X, int64_t ldx );

/*
 * Solve then refine; replaces pastix_task_solve_and_refine
 * (refinement/pastix_task_refine.c:354).  X receives the solution.
 */
PASTIX_GPU_API int pastix_gpu_solve_and_refine( pastix_gpu_t *ctx, int64_t nrhs, const void *B,
                                 int64_t ldb, void *X, int64_t ldx );

/*
 * Independent systems merged into one block-diagonal structure (a batch):
 * segptr[0..nseg] are the first user-numbered unknowns of each system
 * (segptr[0] = 0, segptr[nseg] = n).  CG refinement then stops when every
 * system meets its own test ||r_s||_2 / ||b_s||_2 <= eps (the reference runs
 * each system's refinement separately, refinement/z_refine_grad.c:49), and
 * DPARM_RELATIVE_ERROR reports the largest of them.  nseg = 0 clears it.
 * No reference counterpart: the reference has no batched entry point.
 */
PASTIX_GPU_API int pastix_gpu_set_segments( pastix_gpu_t *ctx, int64_t nseg, const int64_t *segptr );

/*
 * Learned cost model hooks (the reference's cost models, common/models.c,
 * have no GPU counterpart: these are new entry points).
 * pastix_gpu_record_tasks(ctx, 1): the following numfact calls record the
 * device time of every task (one CTA each: a cblk's panel factorization, a
 * TRSM row chunk, an update-GEMM tile).  pastix_gpu_task_records: with info
 * or ns NULL, *count receives the number of records; else up to *count
 * records are written, info[8 r .. 8 r + 7] = {kind (0 panel, 1 TRSM chunk,
 * 2 FMA GEMM tile, 3 tensor-core GEMM tile), cblk, a, b, c, d, element
 * bytes, form (0 LL^t, 1 LU, 2 LDL^t, 3 LDL^h)} with (a, b, c, d) =
 * (w, h, rows solved in the panel kernel, blocks) for a panel,
 * (w, rows, mode, panel) for a TRSM chunk, (K, M, N, flags) for a GEMM tile,
 * and ns[r] its duration in nanoseconds.
 * pastix_gpu_task_times: the same records' start and end stamps (device
 * global timer, ns), times[2 r] and times[2 r + 1], for a timeline.
 * pastix_gpu_set_cblk_priority: predicted cost per cblk; inside each level
 * the panels, TRSM chunks and GEMM tiles of costlier cblks launch first
 * (longest-processing-time order).  NULL restores the cblk order.
 */
PASTIX_GPU_API int pastix_gpu_record_tasks( pastix_gpu_t *ctx, int on );
PASTIX_GPU_API int pastix_gpu_task_records( pastix_gpu_t *ctx, int64_t *count, int64_t *info, double *ns );
PASTIX_GPU_API int pastix_gpu_task_times( pastix_gpu_t *ctx, int64_t *count, int64_t *times );
PASTIX_GPU_API int pastix_gpu_set_cblk_priority( pastix_gpu_t *ctx, const double *prio );

/*
 * Phase timeline of the last numfact that launched its kernels directly (not
 * a graph replay): one record per timed interval, info[3 r .. 3 r + 2] =
 * {stream (0 main, 1 lookahead), phase (0 diagonal blocks, 1 panel TRSM,
 * 2 FMA update GEMMs, 3 tensor-core update GEMMs), elimination-tree level}
 * and times[2 r], times[2 r + 1] its start and end in ms from the start of
 * the numfact (CUDA events).  With info or times NULL, *count receives the
 * number of records; else up to *count are written.  The reference's
 * counterpart is its kernel trace (kernels/kernels_trace.c), which times the
 * CPU kernels.
 */
PASTIX_GPU_API int pastix_gpu_phase_log( pastix_gpu_t *ctx, int64_t *count, int64_t *info, double *times );

/*
 * Kernel variants and launch shapes (the autotuner's knobs, no reference
 * counterpart; the reference's equivalents are compile-time block sizes):
 *   PGPU_TUNE_MIXED_GEMM      0 FP32 FMA, 1 TF32, 2 3xTF32, 3 3xFP16 (default) update GEMMs
 *   PGPU_TUNE_TC_KERNEL       1 persistent warp-specialized (default), 0 one tile per CTA
 *   PGPU_TUNE_LOOKAHEAD       1 (default): deferred update GEMMs on a second stream
 *   PGPU_TUNE_LA_RESERVED_SMS SMs left to the critical path by the second stream (16)
 *   PGPU_TUNE_TRSM_GEMM       1 (default): tall panels' TRSM as a GEMM against the inverse
 *   PGPU_TUNE_TRSM_GEMM_ROWS  panel height above which it applies (256)
 *   PGPU_TUNE_TC_MIN_MN       smallest M x N update sent to the tensor cores (8192)
 *   PGPU_TUNE_WIDE_PANEL      narrowest diagonal block factorized by the 512-thread
 *                             left-looking kernel (128; 0 disables it)
 *   PGPU_TUNE_TC_TMA          1 (default): split operands (3xFP16 / 3xTF32) pre-split once per
 *                             panel and loaded by TMA; 0: 3xTF32 split by producer warps per tile
 *   PGPU_TUNE_TC_PAIR_MIN     TMA kernel: fewest tiles in a launch for pairing 128-row
 *                             tiles that share their B tile (-1, default: 2 per SM)
 *   PGPU_TUNE_DMMA            1 (default): real FP64 update / TRSM GEMMs large enough
 *                             for a 128 x 64 tile on the FP64 tensor cores (DMMA); 0: FMA tiles
 *   PGPU_TUNE_SOLVE_FLOW      1 (default): runs of solve levels whose cblks all hold a
 *                             diagonal-block inverse go through one dataflow launch per
 *                             direction (per-cblk counters instead of per-level launches;
 *                             1, 2 or 4 right-hand sides, complex128: 1 or 2); 0: per-level launches
 *   PGPU_TUNE_GRAPH           -1 (default): the factorization captured as a CUDA graph and
 *                             replayed when the factor holds at most 2^24 coefficients
 *                             (launch-bound sizes); 1 always; 0 never
 * Setting one invalidates the factorization plan (rebuilt by the next numfact).
 */
#define PGPU_TUNE_MIXED_GEMM      0
#define PGPU_TUNE_TC_KERNEL       1
#define PGPU_TUNE_LOOKAHEAD       2
#define PGPU_TUNE_LA_RESERVED_SMS 3
#define PGPU_TUNE_TRSM_GEMM       4
#define PGPU_TUNE_TRSM_GEMM_ROWS  5
#define PGPU_TUNE_TC_MIN_MN       6
#define PGPU_TUNE_WIDE_PANEL      7
#define PGPU_TUNE_TC_TMA          8
#define PGPU_TUNE_TC_PAIR_MIN     9
#define PGPU_TUNE_DMMA            10
#define PGPU_TUNE_SOLVE_FLOW      11
#define PGPU_TUNE_GRAPH           12
#define PGPU_TUNE_COUNT           13
PASTIX_GPU_API int pastix_gpu_set_tuning( pastix_gpu_t *ctx, int key, int64_t value );
PASTIX_GPU_API int pastix_gpu_get_tuning( pastix_gpu_t *ctx, int key, int64_t *value );

/* Copy the output parameters (iparm/dparm, reference indices) out. */
PASTIX_GPU_API int pastix_gpu_get_params( pastix_gpu_t *ctx, int64_t *iparm, double *dparm );
/* Change one parameter between calls (e.g. IPARM_MIXED, IPARM_REFINEMENT). */
PASTIX_GPU_API int pastix_gpu_set_iparm( pastix_gpu_t *ctx, int index, int64_t value );
PASTIX_GPU_API int pastix_gpu_set_dparm( pastix_gpu_t *ctx, int index, double value );

/*
 * Download the factors in the reference's 1D panel layout: cblk after cblk,
 * a column-major stride x width panel whose rows follow the cblk's blocks
 * (the layout of cpucblk_zalloc_fr for a 1D cblk, kernels/cpucblk_zinit.c:220).
 * Element type: the factor type (double/float, complex for Hermitian).
 * U receives U^T for LU (may be NULL otherwise).
 */
PASTIX_GPU_API int pastix_gpu_coeftab( pastix_gpu_t *ctx, void *L, void *U );

/*
 * Launch statistics of the last numfact / solve / refine: number of kernel
 * launches issued and the device time (ms) each phase took.
 *   stats[0] numfact launches, stats[1] solve launches, stats[2] refine launches
 *   stats[3] numfact ms, stats[4] solve ms, stats[5] refine ms
 *   stats[6] update-GEMM ms inside numfact (CUDA events around those launches)
 *   stats[7] update-GEMM launches inside numfact
 *   stats[8] diagonal-factorization ms, stats[9] panel-TRSM ms inside numfact
 *   stats[10] algorithmic flops of the update GEMMs (sum of 2 M N K)
 *   stats[11] ms of the tensor-core update-GEMM launches (part of stats[6]): tcgen05
 *             for single precision, DMMA for real FP64
 *   stats[12] algorithmic flops of the GEMM tasks that ran on the tensor cores
 *   stats[13] tensor-core tiles whose bounded MMA wait timed out (0 when healthy)
 *   stats[14] 1 when the factorization replayed a captured CUDA graph
 *   stats[15] ms of the last pastix_gpu_spm (device-side pattern setup: uploads,
 *             fill map, CSR)
 * (16 doubles)
 * The single-precision (mixed) factorization runs its large update GEMMs on
 * the tensor cores with split FP16 operands (3xFP16); environment
 * PASTIX_GPU_MIXED_GEMM=3xtf32 | tf32 | fp32 selects the 3xTF32 split, one
 * TF32 product, or FMA tiles instead.
 */
PASTIX_GPU_API int pastix_gpu_stats( pastix_gpu_t *ctx, double *stats );

/*
 * Host analysis for a matrix on an nx x ny x nz grid (vertex x + nx*(y + ny*z)):
 * the reference's grid nested dissection (pastixOrderGrid,
 * order/order_grids.c:303) with the personal-ordering analysis that follows
 * it (pastix_subtask_order, _symbfact, _reordering, _blend; the call sequence
 * of example/ordering_grid.c:107-123).  Produces the tables
 * pastix_gpu_structure() takes.  iparm may be NULL (reference defaults);
 * IPARM_MIN/MAX_BLOCKSIZE, IPARM_TASKS2D_WIDTH, IPARM_REORDERING_SPLIT/STOP
 * are read.  colptr/rowptr: 0-based CSC pattern (one triangle or both).
 */
typedef struct pastix_gpu_analysis_s pastix_gpu_analysis_t;
PASTIX_GPU_API int pastix_gpu_analyze_grid( pastix_gpu_analysis_t **an, int64_t nx, int64_t ny, int64_t nz,
                                            int64_t n, const int64_t *colptr, const int64_t *rowptr,
                                            const int64_t *iparm );
/*
 * The same tables read from files instead of computed: the SolverMatrix as
 * the reference's solverSave writes it (blend/solver_io.c:261; the format
 * solverLoad reads back, :45) and the ordering as pastixOrderSave writes it
 * (order/order_io.c:293).  A saved analysis is handed to the GPU layer without
 * running it again (refactorizations of the same pattern; the re-entry of
 * pastix_subtask_bcsc2ctab, sopalin/pastix_task_sopalin.c:213).  Returns
 * PASTIX_GPU_ERR_BADPARAMETER for a missing, malformed or inconsistent file.
 */
PASTIX_GPU_API int pastix_gpu_analysis_load( pastix_gpu_analysis_t **an, const char *solver_file,
                                             const char *order_file );
/* sizes[0..4] = n, cblknbr, bloknbr, brownbr, supernodes of the ordering */
PASTIX_GPU_API int pastix_gpu_analysis_sizes( const pastix_gpu_analysis_t *an, int64_t *sizes );
/* cblktab (cblknbr+1) x 4, bloktab bloknbr x 4, browtab, permtab/peritab (n),
 * rangtab (supernodes+1) and treetab (supernodes) of the ordering; any may be NULL */
PASTIX_GPU_API int pastix_gpu_analysis_export( const pastix_gpu_analysis_t *an, int64_t *cblktab,
                                               int64_t *bloktab, int64_t *browtab, int64_t *permtab,
                                               int64_t *peritab, int64_t *rangtab, int64_t *treetab );
PASTIX_GPU_API void pastix_gpu_analysis_free( pastix_gpu_analysis_t **an );

/*
 * The learned cost model's network: an MLP nfeat -> hidden -> hidden -> 1
 * (ReLU) in FP64, trained and evaluated on the GPU by the library's own
 * kernels (forward, backward, Adam).  Parameters packed as W1[hidden][nfeat],
 * b1[hidden], W2[hidden][hidden], b2[hidden], W3[hidden], b3.  X is row-major
 * n x nfeat (host), targets t and outputs y have n entries; the loss is the
 * mean squared error.  Replaces the offline-fitted polynomial models of
 * common/models.c (no C-ABI counterpart in the reference).
 */
typedef struct pastix_gpu_mlp_s pastix_gpu_mlp_t;
PASTIX_GPU_API int pastix_gpu_mlp_init( pastix_gpu_mlp_t **m, int device, int nfeat, int hidden, uint64_t seed );
PASTIX_GPU_API int pastix_gpu_mlp_params( pastix_gpu_mlp_t *m, double *params, int64_t *count );
PASTIX_GPU_API int pastix_gpu_mlp_set_params( pastix_gpu_mlp_t *m, const double *params );
PASTIX_GPU_API int pastix_gpu_mlp_forward( pastix_gpu_mlp_t *m, int64_t n, const double *X, double *y );
PASTIX_GPU_API int pastix_gpu_mlp_gradient( pastix_gpu_mlp_t *m, int64_t n, const double *X, const double *t,
                                            double *grad, double *loss );
PASTIX_GPU_API int pastix_gpu_mlp_train( pastix_gpu_mlp_t *m, int64_t n, const double *X, const double *t,
                                         int steps, double lr, double *loss );
PASTIX_GPU_API void pastix_gpu_mlp_free( pastix_gpu_mlp_t **m );

/* Release the device memory and the context (pastixFinalize, common/api.c:914). */
PASTIX_GPU_API void pastix_gpu_finalize( pastix_gpu_t **ctx );

#ifdef __cplusplus
}
#endif

#endif /* PASTIX_GPU_H */
