/*
 * Single-process implementations of the SPM routines the PaStiX core calls
 * (see spm.h).  Only the CSC format with a constant dof of 1 is handled,
 * which is all the oracle's synthetic matrices use.  Symmetric and Hermitian
 * matrices hold their lower triangle, as SPM's own generators produce them.
 *
 * Test infrastructure only.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <complex.h>
#include "spm.h"

static size_t elt_size( spm_coeftype_t t )
{
    switch ( t ) {
    case SpmFloat:     return 4;
    case SpmDouble:    return 8;
    case SpmComplex32: return 8;
    case SpmComplex64: return 16;
    default:           return 0;
    }
}

void spmInit( spmatrix_t *spm )
{
    memset( spm, 0, sizeof( *spm ) );
    spm->mtxtype  = SpmGeneral;
    spm->flttype  = SpmDouble;
    spm->fmttype  = SpmCSC;
    spm->dof      = 1;
    spm->layout   = SpmColMajor;
    spm->clustnbr = 1;
    spm->replicated = 1;
}

void spmInitDist( spmatrix_t *spm, SPM_Comm comm )
{
    spmInit( spm );
    spm->comm = comm;
}

void spmExit( spmatrix_t *spm )
{
    free( spm->colptr );
    free( spm->rowptr );
    free( spm->loc2glob );
    free( spm->values );
    free( spm->dofs );
    free( spm->glob2loc );
    spm->colptr = spm->rowptr = spm->loc2glob = spm->dofs = spm->glob2loc = NULL;
    spm->values = NULL;
}

void spmUpdateComputedFields( spmatrix_t *spm )
{
    spm->gN      = spm->n;
    spm->gnnz    = spm->nnz;
    spm->nexp    = spm->n * spm->dof;
    spm->gNexp   = spm->nexp;
    spm->nnzexp  = spm->nnz * spm->dof * spm->dof;
    spm->gnnzexp = spm->nnzexp;
}

spm_int_t spmFindBase( const spmatrix_t *spm )
{
    spm_int_t b = spm->colptr[0];
    for ( spm_int_t k = 0; k < spm->nnz; k++ ) {
        if ( spm->rowptr[k] < b ) {
            b = spm->rowptr[k];
        }
    }
    return b < 0 ? 0 : ( b > 1 ? 1 : b );
}

void spmBase( spmatrix_t *spm, int baseval )
{
    spm_int_t d = baseval - spm->baseval;
    if ( d == 0 ) {
        return;
    }
    for ( spm_int_t j = 0; j <= spm->n; j++ ) {
        spm->colptr[j] += d;
    }
    for ( spm_int_t k = 0; k < spm->nnz; k++ ) {
        spm->rowptr[k] += d;
    }
    if ( spm->loc2glob ) {
        for ( spm_int_t j = 0; j < spm->n; j++ ) {
            spm->loc2glob[j] += d;
        }
    }
    spm->baseval = baseval;
}

static void *dup_mem( const void *p, size_t n )
{
    if ( p == NULL ) {
        return NULL;
    }
    void *q = malloc( n ? n : 1 );
    memcpy( q, p, n );
    return q;
}

void spmCopy( const spmatrix_t *in, spmatrix_t *out )
{
    *out = *in;
    out->colptr   = dup_mem( in->colptr, ( in->n + 1 ) * sizeof( spm_int_t ) );
    out->rowptr   = dup_mem( in->rowptr, in->nnz * sizeof( spm_int_t ) );
    out->loc2glob = dup_mem( in->loc2glob, in->n * sizeof( spm_int_t ) );
    out->values   = dup_mem( in->values, in->nnz * elt_size( in->flttype ) );
    out->dofs     = NULL;
    out->glob2loc = NULL;
}

/* Sort the row indices of every column, carrying the values along. */
int spmSort( spmatrix_t *spm )
{
    size_t es = elt_size( spm->flttype );
    char tmp[16];
    for ( spm_int_t j = 0; j < spm->n; j++ ) {
        spm_int_t s = spm->colptr[j] - spm->baseval, e = spm->colptr[j + 1] - spm->baseval;
        for ( spm_int_t a = s + 1; a < e; a++ ) {
            spm_int_t r = spm->rowptr[a];
            if ( es ) memcpy( tmp, (char *)spm->values + a * es, es );
            spm_int_t b = a - 1;
            while ( b >= s && spm->rowptr[b] > r ) {
                spm->rowptr[b + 1] = spm->rowptr[b];
                if ( es ) memcpy( (char *)spm->values + ( b + 1 ) * es, (char *)spm->values + b * es, es );
                b--;
            }
            spm->rowptr[b + 1] = r;
            if ( es ) memcpy( (char *)spm->values + ( b + 1 ) * es, tmp, es );
        }
    }
    return 0;
}

/*
 * Make the pattern structurally symmetric: every missing transposed entry is
 * added (with a zero value when the matrix carries values).  PaStiX calls it
 * on the value-less graph of Symmetric/Hermitian matrices, which hold one
 * triangle only (graph/graph_prepare.c:144-150).  Returns the number of
 * entries added.
 */
spm_int_t spmSymmetrize( spmatrix_t *spm )
{
    spm_int_t n = spm->n, base = spm->baseval;
    size_t es = elt_size( spm->flttype );
    /* count missing */
    spm_int_t *cnt = calloc( n + 1, sizeof( spm_int_t ) );
    spm_int_t added = 0;
    for ( spm_int_t j = 0; j < n; j++ ) {
        for ( spm_int_t k = spm->colptr[j] - base; k < spm->colptr[j + 1] - base; k++ ) {
            spm_int_t i = spm->rowptr[k] - base;
            if ( i == j ) continue;
            int found = 0;
            for ( spm_int_t l = spm->colptr[i] - base; l < spm->colptr[i + 1] - base; l++ ) {
                if ( spm->rowptr[l] - base == j ) { found = 1; break; }
            }
            if ( !found ) { cnt[i]++; added++; }
        }
    }
    if ( added == 0 ) {
        free( cnt );
        return 0;
    }
    spm_int_t *ncol = malloc( ( n + 1 ) * sizeof( spm_int_t ) );
    ncol[0] = 0;
    for ( spm_int_t j = 0; j < n; j++ ) {
        ncol[j + 1] = ncol[j] + ( spm->colptr[j + 1] - spm->colptr[j] ) + cnt[j];
    }
    spm_int_t *nrow = malloc( ncol[n] * sizeof( spm_int_t ) );
    char *nval = es ? calloc( ncol[n], es ) : NULL;
    spm_int_t *pos = malloc( n * sizeof( spm_int_t ) );
    for ( spm_int_t j = 0; j < n; j++ ) {
        pos[j] = ncol[j];
        for ( spm_int_t k = spm->colptr[j] - base; k < spm->colptr[j + 1] - base; k++ ) {
            nrow[pos[j]] = spm->rowptr[k] - base;
            if ( es ) memcpy( nval + pos[j] * es, (char *)spm->values + k * es, es );
            pos[j]++;
        }
    }
    for ( spm_int_t j = 0; j < n; j++ ) {
        for ( spm_int_t k = spm->colptr[j] - base; k < spm->colptr[j + 1] - base; k++ ) {
            spm_int_t i = spm->rowptr[k] - base;
            if ( i == j ) continue;
            int found = 0;
            for ( spm_int_t l = spm->colptr[i] - base; l < spm->colptr[i + 1] - base; l++ ) {
                if ( spm->rowptr[l] - base == j ) { found = 1; break; }
            }
            if ( !found ) { nrow[pos[i]++] = j; }
        }
    }
    for ( spm_int_t j = 0; j <= n; j++ ) ncol[j] += base;
    for ( spm_int_t k = 0; k < ncol[n] - base; k++ ) nrow[k] += base;
    free( spm->colptr ); free( spm->rowptr ); free( spm->values );
    spm->colptr = ncol; spm->rowptr = nrow; spm->values = nval;
    spm->nnz = ncol[n] - base;
    free( cnt ); free( pos );
    spmUpdateComputedFields( spm );
    spmSort( spm );
    return added;
}

int spmScatter( spmatrix_t *newspm, int root, const spmatrix_t *oldspm, spm_int_t n,
                const spm_int_t *loc2glob, int distByColumn, SPM_Comm comm )
{
    (void)root; (void)n; (void)loc2glob; (void)distByColumn; (void)comm;
    spmCopy( oldspm, newspm );
    return 0;
}

int spmGather( const spmatrix_t *in, int root, spmatrix_t *out )
{
    (void)root;
    if ( out ) spmCopy( in, out );
    return 0;
}

int spmSave( const spmatrix_t *spm, const char *filename )
{
    (void)spm; (void)filename;
    return 1;
}

int spmLoad( spmatrix_t *spm, const char *filename )
{
    (void)spm; (void)filename;
    return 1;
}

/* Value magnitude squared for each arithmetic. */
static double absval( const spmatrix_t *spm, spm_int_t k )
{
    switch ( spm->flttype ) {
    case SpmFloat:     return fabs( ( (float *)spm->values )[k] );
    case SpmDouble:    return fabs( ( (double *)spm->values )[k] );
    case SpmComplex32: return cabsf( ( (float _Complex *)spm->values )[k] );
    case SpmComplex64: return cabs( ( (double _Complex *)spm->values )[k] );
    default:           return 0.;
    }
}

/*
 * Matrix norms of the full matrix.  For Symmetric/Hermitian storage the
 * off-diagonal entries stand for two entries of the matrix.
 */
double spmNorm( spm_normtype_t ntype, const spmatrix_t *spm )
{
    spm_int_t n = spm->n, base = spm->baseval;
    int sym = spm->mtxtype != SpmGeneral;
    if ( ntype == SpmFrobeniusNorm ) {
        /* scaled sum of squares, as LAPACK's lassq */
        double scale = 0., sumsq = 1.;
        for ( spm_int_t j = 0; j < n; j++ ) {
            for ( spm_int_t k = spm->colptr[j] - base; k < spm->colptr[j + 1] - base; k++ ) {
                spm_int_t i = spm->rowptr[k] - base;
                double v = absval( spm, k );
                int mult = ( sym && i != j ) ? 2 : 1;
                if ( v != 0. ) {
                    if ( scale < v ) {
                        sumsq = mult + sumsq * ( scale / v ) * ( scale / v );
                        scale = v;
                    } else {
                        sumsq += mult * ( v / scale ) * ( v / scale );
                    }
                }
            }
        }
        return scale * sqrt( sumsq );
    }
    if ( ntype == SpmMaxNorm ) {
        double m = 0.;
        for ( spm_int_t k = 0; k < spm->nnz; k++ ) {
            double v = absval( spm, k );
            if ( v > m ) m = v;
        }
        return m;
    }
    /* one / inf norms: column or row sums of the full matrix */
    double *acc = calloc( n, sizeof( double ) );
    for ( spm_int_t j = 0; j < n; j++ ) {
        for ( spm_int_t k = spm->colptr[j] - base; k < spm->colptr[j + 1] - base; k++ ) {
            spm_int_t i = spm->rowptr[k] - base;
            double v = absval( spm, k );
            if ( ntype == SpmOneNorm ) acc[j] += v; else acc[i] += v;
            if ( sym && i != j ) {
                if ( ntype == SpmOneNorm ) acc[i] += v; else acc[j] += v;
            }
        }
    }
    double m = 0.;
    for ( spm_int_t j = 0; j < n; j++ ) if ( acc[j] > m ) m = acc[j];
    free( acc );
    return m;
}

int spmExpand( const spmatrix_t *in, spmatrix_t *out )
{
    spmCopy( in, out );
    return 0;
}

int spmConvert( int ofmttype, spmatrix_t *ospm )
{
    return ( ofmttype == (int)ospm->fmttype ) ? 0 : 1;
}

spm_int_t *spm_get_glob2loc( spmatrix_t *spm )
{
    if ( spm->glob2loc == NULL ) {
        spm->glob2loc = malloc( spm->gN * sizeof( spm_int_t ) );
        for ( spm_int_t j = 0; j < spm->gN; j++ ) spm->glob2loc[j] = j;
    }
    return spm->glob2loc;
}

int spmCheckAndCorrect( const spmatrix_t *in, spmatrix_t *out )
{
    (void)in; (void)out;
    return 0;
}

void spmPrintInfo( const spmatrix_t *spm, FILE *stream )
{
    fprintf( stream, "  spm: n=%ld nnz=%ld mtxtype=%d flttype=%d\n", (long)spm->n,
             (long)spm->nnz, (int)spm->mtxtype, (int)spm->flttype );
}
