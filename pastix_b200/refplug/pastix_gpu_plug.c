/*
 * pastix_gpu_plug.c -- the PaStiX-side binding of libpastix_gpu.
 *
 * Compiled into a PaStiX build (it includes PaStiX's internal headers) and
 * linked with the GNU linker option --wrap=<symbol> for every __wrap_<symbol>
 * defined below, it routes the reference's own public API -- pastixInit,
 * pastix_task_analyze, pastix_task_numfact, pastix_task_solve,
 * pastix_task_refine, pastixFinalize, the call sequence of example/simple.c
 * -- into the B200 layer, without changing a line of the PaStiX sources:
 *
 *   plug point (reference)                                  routed to
 *   coeftabInit (sopalin/coeftab.c:204)                     no host coeftab: the device
 *                                                           coeftab is laid out by
 *                                                           pastix_gpu_structure
 *   sopalinFacto[fact][prec] (sopalin/pastix_task_sopalin.c:51-58):
 *     sopalin_{s,d,c,z}potrf / getrf / sytrf, sopalin_{c,z}hetrf
 *                                                           pastix_gpu_numfact
 *   ztrsm_table via sopalin_{s,d,c,z}trsm
 *     (sopalin/sequential_ztrsm.c:536-552,591)              pastix_gpu_solve_steps (one sweep)
 *   zdiag_table via sopalin_{s,d,c,z}diag
 *     (sopalin/sequential_zdiag.c:298,340)                  pastix_gpu_solve_steps (diagonal)
 *   sopalinRefine[refine][prec] (refinement/pastix_task_refine.c:40):
 *     {d,z}_grad_smp, {d,z}_gmres_smp                       pastix_gpu_refine
 *   pastixFinalize (common/api.c:914)                       pastix_gpu_finalize
 *
 * The device state hangs off each pastix_data_t through a small side table
 * (the reference is re-entrant per instance, example/reentrant.c), so no
 * field is added to pastix_data_t (common/pastixdata.h:67-132).  The
 * structure (SolverMatrix, ordering) and the user matrix's pattern are
 * handed over at the first factorization of an analysis; later
 * factorizations of the same pattern only move values.
 *
 * Forms the GPU layer does not provide (LL^t of complex symmetric matrices,
 * dof > 1, matrices in single precision) are left to the reference's own CPU
 * path: their host coeftab is then allocated as usual.
 */
#include "common.h"
#include "blend/solver.h"
#include "bcsc/bcsc.h"
#include "order/order_internal.h"
#include "sopalin/sopalin_data.h"
#include <pastix.h>
#include <pthread.h>
#include <stdio.h>
#include <string.h>

#include "pastix_gpu.h"

/* ------------------------------------------------------------------------ */
/* side table: pastix_data_t -> device context                              */
/* ------------------------------------------------------------------------ */
#define PLUG_MAX 64
typedef struct plug_entry_s {
    pastix_data_t      *pd;
    pastix_gpu_t       *ctx;
    const SolverMatrix *solv;      /* analysis the structure was handed over for */
    const spmatrix_t   *spm;       /* matrix whose pattern was handed over */
    int                 failed;    /* last GPU factorization failed */
} plug_entry_t;

static plug_entry_t    plug_tab[PLUG_MAX];
static pthread_mutex_t plug_lock = PTHREAD_MUTEX_INITIALIZER;

static plug_entry_t *plug_find( pastix_data_t *pd, int create )
{
    plug_entry_t *e = NULL;
    pthread_mutex_lock( &plug_lock );
    for ( int i = 0; i < PLUG_MAX; i++ ) {
        if ( plug_tab[i].pd == pd ) { e = plug_tab + i; break; }
    }
    if ( !e && create ) {
        for ( int i = 0; i < PLUG_MAX; i++ ) {
            if ( plug_tab[i].pd == NULL ) {
                e = plug_tab + i;
                memset( e, 0, sizeof( *e ) );
                e->pd = pd;
                break;
            }
        }
    }
    pthread_mutex_unlock( &plug_lock );
    return e;
}

/* The GPU layer takes int64_t parameters (PaStiX's pastix_int_t with PASTIX_INT64). */
static void plug_params( pastix_data_t *pd, int64_t *ip, double *dp )
{
    for ( int i = 0; i < PGPU_IPARM_SIZE && i < IPARM_SIZE; i++ ) ip[i] = pd->iparm[i];
    for ( int i = 0; i < PGPU_DPARM_SIZE && i < DPARM_SIZE; i++ ) dp[i] = pd->dparm[i];
}

static void plug_sync_params( plug_entry_t *e )
{
    const int ikeys[] = { PGPU_IPARM_FACTORIZATION, PGPU_IPARM_REFINEMENT, PGPU_IPARM_ITERMAX,
                          PGPU_IPARM_GMRES_IM, PGPU_IPARM_MIXED };
    const int dkeys[] = { PGPU_DPARM_EPSILON_REFINEMENT, PGPU_DPARM_EPSILON_MAGN_CTRL };
    for ( size_t i = 0; i < sizeof( ikeys ) / sizeof( ikeys[0] ); i++ )
        pastix_gpu_set_iparm( e->ctx, ikeys[i], e->pd->iparm[ikeys[i]] );
    for ( size_t i = 0; i < sizeof( dkeys ) / sizeof( dkeys[0] ); i++ )
        pastix_gpu_set_dparm( e->ctx, dkeys[i], e->pd->dparm[dkeys[i]] );
}

/* Does the GPU layer factorize what this pastix_data_t asks for? */
static int plug_supported( pastix_data_t *pd )
{
    const spmatrix_t *spm = pd->csc;
    if ( !spm || spm->dof != 1 || pd->solvmatr == NULL ) return 0;
    if ( spm->flttype != SpmDouble && spm->flttype != SpmComplex64 ) return 0;
    if ( pd->iparm[IPARM_FACTORIZATION] == PastixFactLLT && spm->flttype == SpmComplex64 ) return 0;
    return 1;
}

/* SolverMatrix (blend/solver.h:137-273) + ordering -> pastix_gpu_structure,
 * the user's CSC pattern -> pastix_gpu_spm. */
static int plug_handover( plug_entry_t *e )
{
    pastix_data_t      *pd = e->pd;
    const SolverMatrix *s  = pd->solvmatr;
    const spmatrix_t   *A  = pd->csc;
    int                 rc;

    if ( e->solv != s ) {
        const pastix_int_t nc = s->cblknbr, nb = s->bloknbr, n = pd->ordemesh->vertnbr;
        int64_t *cblktab = malloc( 4 * ( nc + 1 ) * sizeof( int64_t ) );
        int64_t *bloktab = malloc( 4 * nb * sizeof( int64_t ) );
        int64_t *browtab = malloc( ( s->brownbr > 0 ? s->brownbr : 1 ) * sizeof( int64_t ) );
        int64_t *perm    = malloc( n * sizeof( int64_t ) );
        int64_t *invp    = malloc( n * sizeof( int64_t ) );
        for ( pastix_int_t c = 0; c <= nc; c++ ) {
            const SolverCblk *cb = s->cblktab + c;
            cblktab[4 * c + 0] = cb->fcolnum;
            cblktab[4 * c + 1] = cb->lcolnum;
            cblktab[4 * c + 2] = cb->fblokptr - s->bloktab;
            cblktab[4 * c + 3] = cb->brownum;
        }
        for ( pastix_int_t b = 0; b < nb; b++ ) {
            const SolverBlok *bk = s->bloktab + b;
            bloktab[4 * b + 0] = bk->frownum;
            bloktab[4 * b + 1] = bk->lrownum;
            bloktab[4 * b + 2] = bk->lcblknm;
            bloktab[4 * b + 3] = bk->fcblknm;
        }
        for ( pastix_int_t i = 0; i < s->brownbr; i++ ) browtab[i] = s->browtab[i];
        for ( pastix_int_t i = 0; i < n; i++ ) {
            perm[i] = pd->ordemesh->permtab[i];
            invp[i] = pd->ordemesh->peritab[i];
        }
        rc = pastix_gpu_structure( e->ctx, n, nc, cblktab, nb, bloktab, s->brownbr, browtab, perm, invp );
        free( cblktab ); free( bloktab ); free( browtab ); free( perm ); free( invp );
        if ( rc ) return rc;
        e->solv = s;
        e->spm  = NULL;
    }
    if ( e->spm != A ) {
        const pastix_int_t n = A->n, nnz = A->nnz, base = A->baseval;
        int64_t *colptr = malloc( ( n + 1 ) * sizeof( int64_t ) );
        int64_t *rowptr = malloc( ( nnz > 0 ? nnz : 1 ) * sizeof( int64_t ) );
        for ( pastix_int_t j = 0; j <= n; j++ ) colptr[j] = A->colptr[j] - base;
        for ( pastix_int_t k = 0; k < nnz; k++ ) rowptr[k] = A->rowptr[k] - base;
        rc = pastix_gpu_spm( e->ctx, A->mtxtype, A->flttype, n, colptr, rowptr );
        free( colptr ); free( rowptr );
        if ( rc ) return rc;
        e->spm = A;
    }
    return PASTIX_SUCCESS;
}

static plug_entry_t *plug_context( pastix_data_t *pd )
{
    plug_entry_t *e = plug_find( pd, 1 );
    if ( !e ) return NULL;
    if ( !e->ctx ) {
        int64_t ip[PGPU_IPARM_SIZE];
        double  dp[PGPU_DPARM_SIZE];
        plug_params( pd, ip, dp );
        if ( pastix_gpu_init( &e->ctx, 0, ip, dp ) != 0 ) {
            e->pd = NULL;
            return NULL;
        }
    }
    plug_sync_params( e );
    return e;
}

/* ------------------------------------------------------------------------ */
/* coeftabInit: the coeftab lives on the device                             */
/* ------------------------------------------------------------------------ */
void __real_coeftabInit( pastix_data_t *pastix_data, pastix_coefside_t side );
void __wrap_coeftabInit( pastix_data_t *pastix_data, pastix_coefside_t side )
{
    if ( !plug_supported( pastix_data ) ) {
        __real_coeftabInit( pastix_data, side );
        return;
    }
    pastix_data->solvmatr->globalalloc = pastix_data->iparm[IPARM_GLOBAL_ALLOCATION];
}

/* ------------------------------------------------------------------------ */
/* sopalinFacto: numerical factorization on the GPU                         */
/* ------------------------------------------------------------------------ */
static void plug_factorize( pastix_data_t *pd, sopalin_data_t *sd )
{
    plug_entry_t *e = plug_context( pd );
    int           rc;
    if ( !e ) {
        pastix_print_error( "pastix_gpu_plug: no GPU context" );
        return;
    }
    rc = plug_handover( e );
    if ( !rc ) rc = pastix_gpu_numfact( e->ctx, pd->csc->values );
    e->failed = rc;
    if ( rc ) {
        pastix_print_error( "pastix_gpu_plug: GPU factorization failed (%d)", rc );
        return;
    }
    {
        int64_t ip[PGPU_IPARM_SIZE];
        double  dp[PGPU_DPARM_SIZE];
        pastix_gpu_get_params( e->ctx, ip, dp );
        sd->solvmtx->nbpivots = ip[PGPU_IPARM_STATIC_PIVOTING];
    }
}

#define PLUG_FACTO( name )                                                   \
    void __wrap_##name( pastix_data_t *pd, sopalin_data_t *sd ) { plug_factorize( pd, sd ); }
PLUG_FACTO( sopalin_spotrf )
PLUG_FACTO( sopalin_dpotrf )
PLUG_FACTO( sopalin_cpotrf )
PLUG_FACTO( sopalin_zpotrf )
PLUG_FACTO( sopalin_sgetrf )
PLUG_FACTO( sopalin_dgetrf )
PLUG_FACTO( sopalin_cgetrf )
PLUG_FACTO( sopalin_zgetrf )
PLUG_FACTO( sopalin_ssytrf )
PLUG_FACTO( sopalin_dsytrf )
PLUG_FACTO( sopalin_csytrf )
PLUG_FACTO( sopalin_zsytrf )
PLUG_FACTO( sopalin_chetrf )
PLUG_FACTO( sopalin_zhetrf )

/* ------------------------------------------------------------------------ */
/* ztrsm_table / zdiag_table: solve steps on the permuted right-hand sides   */
/* ------------------------------------------------------------------------ */
static void plug_steps( pastix_data_t *pd, int steps, pastix_int_t nrhs, void *b, pastix_int_t ldb,
                        pastix_coeftype_t flttype )
{
    plug_entry_t *e = plug_find( pd, 0 );
    int           rc;
    if ( !e || !e->ctx || e->failed ) {
        pastix_print_error( "pastix_gpu_plug: solve without a GPU factorization" );
        return;
    }
    rc = pastix_gpu_solve_steps( e->ctx, steps, nrhs, b, ldb, (int)flttype );
    if ( rc ) pastix_print_error( "pastix_gpu_plug: GPU solve step failed (%d)", rc );
}

/* Which sweep a sopalin_ztrsm call is: the lower one (L y = b) or the upper
 * one (L^t, L^h or U), as pastix_subtask_solve_adv issues them. */
static int plug_sweep( pastix_side_t side, pastix_uplo_t uplo, pastix_trans_t trans )
{
    if ( side != PastixLeft ) return 0;
    if ( uplo == PastixLower ) return trans == PastixNoTrans ? PGPU_SOLVE_FORWARD : PGPU_SOLVE_BACKWARD;
    return trans == PastixNoTrans ? PGPU_SOLVE_BACKWARD : 0;
}

#define PLUG_TRSM( name )                                                                  \
    void __real_##name( pastix_data_t *, pastix_side_t, pastix_uplo_t, pastix_trans_t,     \
                        pastix_diag_t, sopalin_data_t *, pastix_rhs_t );                   \
    void __wrap_##name( pastix_data_t *pd, pastix_side_t side, pastix_uplo_t uplo,         \
                        pastix_trans_t trans, pastix_diag_t diag, sopalin_data_t *sd,      \
                        pastix_rhs_t rhsb )                                                \
    {                                                                                      \
        plug_entry_t *e = plug_find( pd, 0 );                                              \
        const int     sw = plug_sweep( side, uplo, trans );                                \
        if ( !e || !e->ctx ) { /* a CPU-factorized form */                                 \
            __real_##name( pd, side, uplo, trans, diag, sd, rhsb );                        \
            return;                                                                        \
        }                                                                                  \
        if ( !sw ) {                                                                       \
            pastix_print_error( "pastix_gpu_plug: triangular solve form not provided" );  \
            return;                                                                        \
        }                                                                                  \
        plug_steps( pd, sw, rhsb->n, rhsb->b, rhsb->ld, rhsb->flttype );                   \
        (void)diag;                                                                        \
    }
PLUG_TRSM( sopalin_strsm )
PLUG_TRSM( sopalin_dtrsm )
PLUG_TRSM( sopalin_ctrsm )
PLUG_TRSM( sopalin_ztrsm )

#define PLUG_DIAG( name, type, flt )                                                       \
    void __real_##name( pastix_data_t *, sopalin_data_t *, int, type *, int );             \
    void __wrap_##name( pastix_data_t *pd, sopalin_data_t *sd, int nrhs, type *b, int ldb ) \
    {                                                                                      \
        plug_entry_t *e = plug_find( pd, 0 );                                              \
        if ( !e || !e->ctx ) {                                                             \
            __real_##name( pd, sd, nrhs, b, ldb );                                         \
            return;                                                                        \
        }                                                                                  \
        plug_steps( pd, PGPU_SOLVE_DIAG, nrhs, b, ldb, flt );                              \
    }
PLUG_DIAG( sopalin_sdiag, float, PastixFloat )
PLUG_DIAG( sopalin_ddiag, double, PastixDouble )
PLUG_DIAG( sopalin_cdiag, pastix_complex32_t, PastixComplex32 )
PLUG_DIAG( sopalin_zdiag, pastix_complex64_t, PastixComplex64 )

/* ------------------------------------------------------------------------ */
/* sopalinRefine: CG / GMRES refinement on the GPU                          */
/* ------------------------------------------------------------------------ */
/* One right-hand side (the reference refines them one after the other,
 * refinement/pastix_task_refine.c:144-165), in the permuted numbering: taken
 * back to the user's numbering for pastix_gpu_refine, which multiplies by the
 * user's matrix and solves with the factors, and permuted again. */
static pastix_int_t plug_refine( pastix_data_t *pd, pastix_rhs_t xp, pastix_rhs_t bp, size_t es )
{
    plug_entry_t *e = plug_find( pd, 0 );
    const pastix_int_t n = bp->m;
    const pastix_int_t *perm = pd->ordemesh->permtab;
    char *x, *b;
    int   rc;
    int64_t ip[PGPU_IPARM_SIZE];
    double  dp[PGPU_DPARM_SIZE];

    if ( !e || !e->ctx || e->failed ) {
        pastix_print_error( "pastix_gpu_plug: refinement without a GPU factorization" );
        return -1;
    }
    plug_sync_params( e );
    x = malloc( n * es );
    b = malloc( n * es );
    for ( pastix_int_t i = 0; i < n; i++ ) {
        memcpy( b + i * es, (char *)bp->b + perm[i] * es, es );
        memcpy( x + i * es, (char *)xp->b + perm[i] * es, es );
    }
    rc = pastix_gpu_refine( e->ctx, 1, b, n, x, n );
    if ( !rc ) {
        for ( pastix_int_t i = 0; i < n; i++ ) memcpy( (char *)xp->b + perm[i] * es, x + i * es, es );
    }
    free( x );
    free( b );
    if ( rc ) {
        pastix_print_error( "pastix_gpu_plug: GPU refinement failed (%d)", rc );
        return -1;
    }
    pastix_gpu_get_params( e->ctx, ip, dp );
    pd->dparm[DPARM_RELATIVE_ERROR] = dp[PGPU_DPARM_RELATIVE_ERROR];
    return ip[PGPU_IPARM_NBITER];
}

#define PLUG_REFINE( name, es )                                                            \
    pastix_int_t __real_##name( pastix_data_t *, pastix_rhs_t, pastix_rhs_t );             \
    pastix_int_t __wrap_##name( pastix_data_t *pd, pastix_rhs_t xp, pastix_rhs_t bp )      \
    {                                                                                      \
        plug_entry_t *e = plug_find( pd, 0 );                                              \
        if ( !e || !e->ctx ) return __real_##name( pd, xp, bp );                           \
        return plug_refine( pd, xp, bp, es );                                              \
    }
PLUG_REFINE( d_grad_smp, sizeof( double ) )
PLUG_REFINE( z_grad_smp, sizeof( pastix_complex64_t ) )
PLUG_REFINE( d_gmres_smp, sizeof( double ) )
PLUG_REFINE( z_gmres_smp, sizeof( pastix_complex64_t ) )

/* ------------------------------------------------------------------------ */
/* pastixFinalize: release the device context with the instance             */
/* ------------------------------------------------------------------------ */
void __real_pastixFinalize( pastix_data_t **pastix_data );
void __wrap_pastixFinalize( pastix_data_t **pastix_data )
{
    plug_entry_t *e = pastix_data ? plug_find( *pastix_data, 0 ) : NULL;
    if ( e ) {
        if ( e->ctx ) pastix_gpu_finalize( &e->ctx );
        pthread_mutex_lock( &plug_lock );
        memset( e, 0, sizeof( *e ) );
        pthread_mutex_unlock( &plug_lock );
    }
    __real_pastixFinalize( pastix_data );
}
