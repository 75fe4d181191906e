/*
 * ctypes-callable driver around the PaStiX reference's public API, used as a
 * test oracle and as the timed CPU baseline.  The call sequence follows the
 * reference's example/ordering_grid.c:107-123 (pastixOrderGrid + personal
 * ordering + the analysis subtasks) and example/simple.c (numfact, solve,
 * refine).  Besides running the reference, it exports what the reference
 * computed: the ordering, the SolverMatrix structure (blend/solver.h:137-273)
 * flattened to integer tables, the factor coeftab, and the bcsc.
 *
 * Test infrastructure only.
 */
#include "common.h"
#include "blend/solver.h"
#include "bcsc/bcsc.h"
#include "order/order_internal.h"
#include <pastix.h>
#include <string.h>

typedef struct ref_handle_s {
    pastix_data_t *pd;
    pastix_int_t   iparm[IPARM_SIZE];
    double         dparm[DPARM_SIZE];
    spmatrix_t     spm;
    int            has_spm;
} ref_handle_t;

/* OpenBLAS entry point: PaStiX requires a sequential BLAS (README.md:76-77);
 * the bundled OpenBLAS is the pthreads build, so pin it to one thread. */
void openblas_set_num_threads( int );

ref_handle_t *ref_create( int nthreads, int verbose )
{
    openblas_set_num_threads( 1 );
    ref_handle_t *h = calloc( 1, sizeof( ref_handle_t ) );
    pastixInitParam( h->iparm, h->dparm );
    h->iparm[IPARM_VERBOSE]    = verbose;
    h->iparm[IPARM_THREAD_NBR] = nthreads;
    h->iparm[IPARM_SCHEDULER]  = PastixSchedStatic;
    spmInit( &h->spm );
    return h;
}

void ref_set_iparm( ref_handle_t *h, int idx, int64_t v ) { h->iparm[idx] = v; }
void ref_set_dparm( ref_handle_t *h, int idx, double v ) { h->dparm[idx] = v; }
int64_t ref_get_iparm( ref_handle_t *h, int idx ) { return h->iparm[idx]; }
double ref_get_dparm( ref_handle_t *h, int idx ) { return h->dparm[idx]; }

/* Starts the library (isched threads) once the parameters are set. */
int ref_init( ref_handle_t *h )
{
    pastixInit( &h->pd, MPI_COMM_WORLD, h->iparm, h->dparm );
    return h->pd ? 0 : 1;
}

/*
 * Hand a 0-based CSC matrix to the handle (copied).  mtxtype uses the
 * reference's values (SpmGeneral/SpmSymmetric/SpmHermitian), flttype its
 * arithmetic codes; symmetric and Hermitian matrices pass their lower
 * triangle.
 */
int ref_set_matrix( ref_handle_t *h, int mtxtype, int flttype, int64_t n,
                    const int64_t *colptr, const int64_t *rowptr, const void *values )
{
    spmatrix_t *spm = &h->spm;
    spmInit( spm );
    spm->mtxtype = mtxtype;
    spm->flttype = flttype;
    spm->fmttype = SpmCSC;
    spm->baseval = 0;
    spm->n       = n;
    spm->nnz     = colptr[n];
    spm->dof     = 1;
    spm->colptr  = malloc( ( n + 1 ) * sizeof( spm_int_t ) );
    spm->rowptr  = malloc( spm->nnz * sizeof( spm_int_t ) );
    memcpy( spm->colptr, colptr, ( n + 1 ) * sizeof( spm_int_t ) );
    memcpy( spm->rowptr, rowptr, spm->nnz * sizeof( spm_int_t ) );
    size_t es = pastix_size_of( flttype );
    spm->values = malloc( spm->nnz * es );
    memcpy( spm->values, values, spm->nnz * es );
    spmUpdateComputedFields( spm );
    h->has_spm = 1;
    return 0;
}

/* Analysis with the reference's Scotch-free grid nested dissection. */
int ref_analyze_grid( ref_handle_t *h, int64_t nx, int64_t ny, int64_t nz )
{
    pastix_order_t *ord = malloc( sizeof( pastix_order_t ) );
    memset( ord, 0, sizeof( pastix_order_t ) );
    int rc = pastixOrderGrid( &ord, nx, ny, nz );
    if ( rc ) return rc;
    h->iparm[IPARM_ORDERING] = PastixOrderPersonal;
    rc = pastix_subtask_order( h->pd, &h->spm, ord );
    if ( rc ) return rc;
    rc = pastix_subtask_symbfact( h->pd );
    if ( rc ) return rc;
    rc = pastix_subtask_reordering( h->pd );
    if ( rc ) return rc;
    rc = pastix_subtask_blend( h->pd );
    pastixOrderExit( ord );
    free( ord );
    return rc;
}

int ref_numfact( ref_handle_t *h ) { return pastix_task_numfact( h->pd, &h->spm ); }

int ref_solve( ref_handle_t *h, int64_t nrhs, void *B, int64_t ldb )
{
    return pastix_task_solve( h->pd, h->spm.n, nrhs, B, ldb );
}

int ref_refine( ref_handle_t *h, int64_t nrhs, void *B, int64_t ldb, void *X, int64_t ldx )
{
    return pastix_task_refine( h->pd, h->spm.n, nrhs, B, ldb, X, ldx );
}

/*
 * Sizes of the exported tables:
 * out[0]=cblknbr out[1]=bloknbr out[2]=brownbr out[3]=coefnbr out[4]=nodenbr
 * out[5]=gemmmax out[6]=offdmax out[7]=blokmax out[8]=colmax out[9]=factotype
 * out[10]=flttype out[11]=nb2dcblk out[12]=cblkmin2d out[13]=cblkmax1d
 */
/*
 * Save the analysis: the SolverMatrix by the reference's own solverSave
 * (blend/solver_io.c:261) into solver_path, and the ordering into order_path
 * in the format of the reference's ordering_save (order/order_io.c:199:
 * "1", cblknbr, vertnbr, then rangtab, permtab and treetab, eight values per
 * line).  The reference's pastixOrderSave (order/order_io.c:293) writes only
 * when pastix_data->procnbr == 0, the total number of processes, which is
 * never the case, so its format is written here.
 */
int ref_save_structure( ref_handle_t *h, const char *solver_path, const char *order_path )
{
    FILE *f = fopen( solver_path, "w" );
    if ( !f ) return 1;
    int rc = solverSave( h->pd->solvmatr, f );
    fclose( f );
    if ( rc ) return rc;
    const pastix_order_t *o = h->pd->ordemesh;
    f = fopen( order_path, "w" );
    if ( !f ) return 1;
    fprintf( f, "1\n%ld\t%ld\n", (long)o->cblknbr, (long)o->vertnbr );
    for ( pastix_int_t k = 0; k <= o->cblknbr; k++ )
        fprintf( f, "%ld%c", (long)o->rangtab[k], ( ( k & 7 ) == 7 || k == o->cblknbr ) ? '\n' : '\t' );
    for ( pastix_int_t k = 0; k < o->vertnbr; k++ )
        fprintf( f, "%ld%c", (long)o->permtab[k], ( ( k & 7 ) == 7 || k == o->vertnbr - 1 ) ? '\n' : '\t' );
    for ( pastix_int_t k = 0; k < o->cblknbr; k++ )
        fprintf( f, "%ld%c", (long)o->treetab[k], ( ( k & 7 ) == 7 || k == o->cblknbr - 1 ) ? '\n' : '\t' );
    fclose( f );
    return 0;
}

int ref_struct_sizes( ref_handle_t *h, int64_t *out )
{
    SolverMatrix *s = h->pd->solvmatr;
    if ( !s ) return 1;
    out[0]  = s->cblknbr;
    out[1]  = s->bloknbr;
    out[2]  = s->brownbr;
    out[3]  = s->coefnbr;
    out[4]  = s->nodenbr;
    out[5]  = s->gemmmax;
    out[6]  = s->offdmax;
    out[7]  = s->blokmax;
    out[8]  = s->colmax;
    out[9]  = s->factotype;
    out[10] = s->flttype;
    out[11] = s->nb2dcblk;
    out[12] = s->cblkmin2d;
    out[13] = s->cblkmax1d;
    return 0;
}

#define REF_NC 10
#define REF_NB 8

/*
 * cblk table (cblknbr+1 rows of REF_NC): fcolnum, lcolnum, first blok index,
 * stride, lcolidx, brownum, brown2d, cblktype, sndeidx, bcscnum.
 * blok table (bloknbr+1 rows of REF_NB): lcblknm, fcblknm, frownum, lrownum,
 * coefind, browind, inlast, iluklvl.
 */
int ref_struct_dump( ref_handle_t *h, int64_t *cblk, int64_t *blok, int64_t *brow,
                     int64_t *perm, int64_t *invp )
{
    SolverMatrix *s = h->pd->solvmatr;
    for ( pastix_int_t c = 0; c <= s->cblknbr; c++ ) {
        SolverCblk *cb = s->cblktab + c;
        int64_t *o = cblk + REF_NC * c;
        o[0] = cb->fcolnum;
        o[1] = cb->lcolnum;
        o[2] = cb->fblokptr - s->bloktab;
        o[3] = cb->stride;
        o[4] = cb->lcolidx;
        o[5] = cb->brownum;
        o[6] = cb->brown2d;
        o[7] = cb->cblktype;
        o[8] = cb->sndeidx;
        o[9] = cb->bcscnum;
    }
    for ( pastix_int_t b = 0; b <= s->bloknbr; b++ ) {
        SolverBlok *bk = s->bloktab + b;
        int64_t *o = blok + REF_NB * b;
        o[0] = bk->lcblknm;
        o[1] = bk->fcblknm;
        o[2] = bk->frownum;
        o[3] = bk->lrownum;
        o[4] = bk->coefind;
        o[5] = bk->browind;
        o[6] = bk->inlast;
        o[7] = bk->iluklvl;
    }
    for ( pastix_int_t i = 0; i < s->brownbr; i++ ) brow[i] = s->browtab[i];
    pastix_order_t *o = h->pd->ordemesh;
    if ( perm && invp && o ) {
        for ( pastix_int_t i = 0; i < o->vertnbr; i++ ) {
            perm[i] = o->permtab[i];
            invp[i] = o->peritab[i];
        }
    }
    return 0;
}

/* Number of supernodes in the ordering and its rangtab/treetab. */
int64_t ref_order_cblknbr( ref_handle_t *h ) { return h->pd->ordemesh->cblknbr; }
int ref_order_dump( ref_handle_t *h, int64_t *rang, int64_t *tree )
{
    pastix_order_t *o = h->pd->ordemesh;
    for ( pastix_int_t i = 0; i <= o->cblknbr; i++ ) rang[i] = o->rangtab[i];
    for ( pastix_int_t i = 0; i < o->cblknbr; i++ ) tree[i] = o->treetab[i];
    return 0;
}

/*
 * Copy the factor panels, cblk after cblk, each stride x width elements as
 * stored (column-major, 1D or 2D layout).  U may be NULL.
 */
int ref_coeftab_dump( ref_handle_t *h, void *L, void *U )
{
    SolverMatrix *s = h->pd->solvmatr;
    size_t es = pastix_size_of( s->flttype );
    size_t off = 0;
    for ( pastix_int_t c = 0; c < s->cblknbr; c++ ) {
        SolverCblk *cb = s->cblktab + c;
        size_t cnt = (size_t)cb->stride * ( cb->lcolnum - cb->fcolnum + 1 );
        if ( L && cb->lcoeftab ) memcpy( (char *)L + off * es, cb->lcoeftab, cnt * es );
        if ( U && cb->ucoeftab ) memcpy( (char *)U + off * es, cb->ucoeftab, cnt * es );
        off += cnt;
    }
    return 0;
}

void ref_destroy( ref_handle_t *h )
{
    if ( h->pd ) pastixFinalize( &h->pd );
    if ( h->has_spm ) spmExit( &h->spm );
    free( h );
}

/*
 * common/isched_nohwloc.c calls pastix_warning(), which no reference source
 * defines (it only links in hwloc-less builds).  Provided here so the
 * no-hwloc scheduler links.
 */
#include <stdarg.h>
void pastix_warning( const char *fmt, ... )
{
    va_list ap;
    va_start( ap, fmt );
    fprintf( stderr, "pastix warning: " );
    vfprintf( stderr, fmt, ap );
    fprintf( stderr, "\n" );
    va_end( ap );
}
