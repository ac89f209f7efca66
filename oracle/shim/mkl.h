/*
 * Test infrastructure (oracle): a minimal stand-in for the Intel oneMKL API surface
 * that the LPM-CPP reference headers call.  MKL is not installed on this machine, so
 * the reference is compiled against these declarations and linked with mkl_shim.cpp.
 *
 * Only the entry points the reference uses are declared (call sites in the reference):
 *   cblas_dnrm2   include/solver.h:63-64,85, include/stiffness.h:378
 *   cblas_dgemm   include/particle_elastic.h:88-90,120-122, include/particle_j2plasticity.h:177-180
 *   cblas_dgemv   include/utilities.h:113,165,205,297
 *   mkl_sparse_d_create_csr / mkl_sparse_d_mv   include/solver.h:284-296,334
 *   dcg_init / dcg_check / dcg / dcg_get        include/solver.h:303-344
 *   PARDISO                                     include/solver.h:238-268
 *   mkl_free_buffers                            src/lpmcpp.cpp:53
 * The semantics follow Intel's public API documentation; the implementations are
 * plain textbook algorithms written for this project (no MKL code).
 */
#pragma once
#ifndef LPM_ORACLE_MKL_SHIM_H
#define LPM_ORACLE_MKL_SHIM_H

#include <climits>
#include <cstdint>

#ifdef MKL_ILP64
typedef long long MKL_INT;
#else
typedef int MKL_INT;
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

double cblas_dnrm2(const MKL_INT n, const double *x, const MKL_INT incx);
void cblas_dgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                 const MKL_INT m, const MKL_INT n, const MKL_INT k, const double alpha,
                 const double *a, const MKL_INT lda, const double *b, const MKL_INT ldb,
                 const double beta, double *c, const MKL_INT ldc);
void cblas_dgemv(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE trans, const MKL_INT m, const MKL_INT n,
                 const double alpha, const double *a, const MKL_INT lda, const double *x, const MKL_INT incx,
                 const double beta, double *y, const MKL_INT incy);

/* sparse BLAS (inspector-executor) */
typedef enum { SPARSE_STATUS_SUCCESS = 0, SPARSE_STATUS_NOT_INITIALIZED = 1, SPARSE_STATUS_INVALID_VALUE = 3,
               SPARSE_STATUS_NOT_SUPPORTED = 6 } sparse_status_t;
typedef enum { SPARSE_OPERATION_NON_TRANSPOSE = 10, SPARSE_OPERATION_TRANSPOSE = 11,
               SPARSE_OPERATION_CONJUGATE_TRANSPOSE = 12 } sparse_operation_t;
typedef enum { SPARSE_MATRIX_TYPE_GENERAL = 20, SPARSE_MATRIX_TYPE_SYMMETRIC = 21 } sparse_matrix_type_t;
typedef enum { SPARSE_FILL_MODE_LOWER = 40, SPARSE_FILL_MODE_UPPER = 41, SPARSE_FILL_MODE_FULL = 42 } sparse_fill_mode_t;
typedef enum { SPARSE_DIAG_NON_UNIT = 50, SPARSE_DIAG_UNIT = 51 } sparse_diag_type_t;
typedef enum { SPARSE_INDEX_BASE_ZERO = 0, SPARSE_INDEX_BASE_ONE = 1 } sparse_index_base_t;

struct matrix_descr
{
    sparse_matrix_type_t type;
    sparse_fill_mode_t mode;
    sparse_diag_type_t diag;
};

struct lpm_shim_sparse_matrix;
typedef struct lpm_shim_sparse_matrix *sparse_matrix_t;

sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *A, const sparse_index_base_t indexing, const MKL_INT rows,
                                        const MKL_INT cols, MKL_INT *rows_start, MKL_INT *rows_end,
                                        MKL_INT *col_indx, double *values);
sparse_status_t mkl_sparse_d_mv(const sparse_operation_t operation, const double alpha, const sparse_matrix_t A,
                                const struct matrix_descr descr, const double *x, const double beta, double *y);
sparse_status_t mkl_sparse_destroy(sparse_matrix_t A);

/* RCI conjugate gradient */
void dcg_init(const MKL_INT *n, const double *x, const double *b, MKL_INT *rci_request, MKL_INT *ipar,
              double *dpar, double *tmp);
void dcg_check(const MKL_INT *n, const double *x, const double *b, MKL_INT *rci_request, MKL_INT *ipar,
               double *dpar, double *tmp);
void dcg(const MKL_INT *n, double *x, double *b, MKL_INT *rci_request, MKL_INT *ipar, double *dpar, double *tmp);
void dcg_get(const MKL_INT *n, const double *x, const double *b, const MKL_INT *rci_request, const MKL_INT *ipar,
             const double *dpar, const double *tmp, MKL_INT *itercount);

/* direct sparse solver */
void PARDISO(void *pt, const MKL_INT *maxfct, const MKL_INT *mnum, const MKL_INT *mtype, const MKL_INT *phase,
             const MKL_INT *n, const void *a, const MKL_INT *ia, const MKL_INT *ja, MKL_INT *perm,
             const MKL_INT *nrhs, MKL_INT *iparm, const MKL_INT *msglvl, void *b, void *x, MKL_INT *error);

void mkl_free_buffers(void);

/* Counters kept by the shim so the oracle driver can report linear-solver work. */
extern "C" {
struct lpm_shim_stats
{
    long long cg_solves;      /* dcg_init calls (one per linear solve) */
    long long cg_iterations;  /* total CG iterations over all solves */
    long long spmv_calls;     /* mkl_sparse_d_mv calls */
    double spmv_seconds;      /* wall time inside mkl_sparse_d_mv */
    double cg_seconds;        /* wall time inside dcg (vector work) */
    double create_seconds;    /* wall time inside mkl_sparse_d_create_csr */
    long long cg_failures;    /* dcg returned a negative request */
    long long cg_maxit_override; /* if > 0, caps ipar[4] at this value (bounded CPU samples) */
    double cg_rtol_override;     /* if >= 0, replaces dpar[0] at dcg_check (tightened parity runs) */
    double cg_atol_override;     /* if >= 0, replaces dpar[1] at dcg_check */
};
extern struct lpm_shim_stats lpm_shim_stats_g;
}

#endif
