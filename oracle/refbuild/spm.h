/*
 * Minimal stand-in for the SPM sparse-matrix library (the reference's `spm/`
 * git submodule, which is empty in the reference tree).  It declares only the
 * types, enumerations and the handful of single-process routines that the
 * PaStiX core library calls (graph/graph.c, order/pastix_subtask_order.c,
 * bcsc/bvec_zlapmr.c, sopalin/pastix.c, sopalin/pastix_task_sopalin.c:118).
 * Enumeration values follow the published SPM interface so that PaStiX's own
 * aliases (include/pastix/api.h:296-302, 457-460) keep their meaning.
 *
 * Test infrastructure only (used to build the reference as an oracle).
 */
#ifndef _spm_h_
#define _spm_h_

#include <stdint.h>
#include <stdio.h>
#include <complex.h>

#include "pastix/config.h"

#if defined(PASTIX_INT64)
typedef int64_t spm_int_t;
#else
typedef int spm_int_t;
#endif

typedef float  _Complex spm_complex32_t;
typedef double _Complex spm_complex64_t;

typedef int SPM_Comm;

#define SPM_SUCCESS        0
#define SPM_ERR_BADPARAMETER 7

typedef enum spm_coeftype_e {
    SpmPattern   = 0,
    SpmFloat     = 2,
    SpmDouble    = 3,
    SpmComplex32 = 4,
    SpmComplex64 = 5
} spm_coeftype_t;

typedef enum spm_fmttype_e {
    SpmCSC = 0,
    SpmCSR = 1,
    SpmIJV = 2
} spm_fmttype_t;

typedef enum spm_mtxtype_e {
    SpmGeneral   = 111,
    SpmSymmetric = 112,
    SpmHermitian = 113
} spm_mtxtype_t;

typedef enum spm_layout_e {
    SpmRowMajor = 101,
    SpmColMajor = 102
} spm_layout_t;

typedef enum spm_normtype_e {
    SpmOneNorm       = 171,
    SpmFrobeniusNorm = 174,
    SpmInfNorm       = 175,
    SpmMaxNorm       = 177
} spm_normtype_t;

typedef enum spm_driver_e {
    SpmDriverRSA,
    SpmDriverHB,
    SpmDriverIJV,
    SpmDriverMM,
    SpmDriverLaplacian,
    SpmDriverXLaplacian,
    SpmDriverGraph,
    SpmDriverSPM
} spm_driver_t;

typedef enum spm_rhstype_e {
    SpmRhsOne,
    SpmRhsI,
    SpmRhsRndX,
    SpmRhsRndB
} spm_rhstype_t;

typedef struct spmatrix_s {
    spm_mtxtype_t  mtxtype;
    spm_coeftype_t flttype;
    spm_fmttype_t  fmttype;
    spm_int_t      baseval;
    spm_int_t      gN;
    spm_int_t      n;
    spm_int_t      gnnz;
    spm_int_t      nnz;
    spm_int_t      gNexp;
    spm_int_t      nexp;
    spm_int_t      gnnzexp;
    spm_int_t      nnzexp;
    spm_int_t      dof;
    spm_int_t     *dofs;
    spm_layout_t   layout;
    spm_int_t     *colptr;
    spm_int_t     *rowptr;
    spm_int_t     *loc2glob;
    void          *values;
    spm_int_t     *glob2loc;
    int            clustnum;
    int            clustnbr;
    int            replicated;
    SPM_Comm       comm;
} spmatrix_t;

void       spmInit( spmatrix_t *spm );
void       spmInitDist( spmatrix_t *spm, SPM_Comm comm );
void       spmExit( spmatrix_t *spm );
void       spmUpdateComputedFields( spmatrix_t *spm );
spm_int_t  spmFindBase( const spmatrix_t *spm );
void       spmBase( spmatrix_t *spm, int baseval );
void       spmCopy( const spmatrix_t *spmin, spmatrix_t *spmout );
int        spmSort( spmatrix_t *spm );
spm_int_t  spmSymmetrize( spmatrix_t *spm );
int        spmScatter( spmatrix_t *newspm, int root, const spmatrix_t *oldspm,
                       spm_int_t n, const spm_int_t *loc2glob, int distByColumn,
                       SPM_Comm comm );
int        spmGather( const spmatrix_t *spm_scattered, int root, spmatrix_t *spm_gathered );
int        spmSave( const spmatrix_t *spm, const char *filename );
int        spmLoad( spmatrix_t *spm, const char *filename );
double     spmNorm( spm_normtype_t ntype, const spmatrix_t *spm );
int        spmExpand( const spmatrix_t *spm_in, spmatrix_t *spm_out );
int        spmConvert( int ofmttype, spmatrix_t *ospm );
spm_int_t *spm_get_glob2loc( spmatrix_t *spm );
int        spmCheckAndCorrect( const spmatrix_t *spm_in, spmatrix_t *spm_out );
void       spmPrintInfo( const spmatrix_t *spm, FILE *stream );

#endif /* _spm_h_ */
