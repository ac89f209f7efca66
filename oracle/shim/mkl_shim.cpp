/*
 * Test infrastructure (oracle): implementations of the MKL entry points declared in mkl.h,
 * written from Intel's public API descriptions as plain textbook algorithms.
 *
 *  - cblas_dnrm2: sqrt of the in-order sum of squares (no scaling pass).
 *  - cblas_dgemm / cblas_dgemv: row-major, no-transpose only (the only forms the reference
 *    uses); each output is alpha * (in-order dot product) + beta * old value (beta term
 *    skipped when beta == 0).
 *  - mkl_sparse_d_create_csr + mkl_sparse_d_mv: the reference passes a 1-based upper-triangular
 *    CSR with a SYMMETRIC/UPPER descriptor (include/solver.h:287-296).  The handle references the
 *    caller's arrays; the product reads the upper triangle once (OpenMP, per-thread scatter
 *    buffers for the transposed half).  The reference never destroys its handles (solver.h:296);
 *    with no copy inside, that leaks only the small handle, as with MKL.
 *  - dcg_*: the RCI state machine of unpreconditioned Hestenes-Stiefel CG.  With ipar[8] != 0
 *    the residual test is ||r||^2 <= dpar[0] * ||r0||^2 + dpar[1] (squared norms, as the
 *    public documentation of dpar[2..4] states); ipar[4] is the iteration cap, ipar[3] the
 *    iteration counter.
 *  - PARDISO: mtype 2 (SPD) stand-in solving by CG to ||r|| <= 1e-14 ||b||.
 */
#include "mkl.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
struct lpm_shim_stats lpm_shim_stats_g = {0, 0, 0, 0.0, 0.0, 0.0, 0, 0, -1.0, -1.0};
}

static double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

double cblas_dnrm2(const MKL_INT n, const double *x, const MKL_INT incx)
{
    double s = 0.0;
    for (MKL_INT i = 0; i < n; ++i)
        s += x[i * incx] * x[i * incx];
    return std::sqrt(s);
}

void cblas_dgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                 const MKL_INT m, const MKL_INT n, const MKL_INT k, const double alpha,
                 const double *a, const MKL_INT lda, const double *b, const MKL_INT ldb,
                 const double beta, double *c, const MKL_INT ldc)
{
    if (layout != CblasRowMajor || transa != CblasNoTrans || transb != CblasNoTrans)
    {
        std::fprintf(stderr, "mkl shim: cblas_dgemm only supports row-major no-transpose\n");
        return;
    }
    for (MKL_INT i = 0; i < m; ++i)
        for (MKL_INT j = 0; j < n; ++j)
        {
            double s = 0.0;
            for (MKL_INT l = 0; l < k; ++l)
                s += a[i * lda + l] * b[l * ldb + j];
            double v = alpha * s;
            if (beta != 0.0)
                v += beta * c[i * ldc + j];
            c[i * ldc + j] = v;
        }
}

void cblas_dgemv(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE trans, const MKL_INT m, const MKL_INT n,
                 const double alpha, const double *a, const MKL_INT lda, const double *x, const MKL_INT incx,
                 const double beta, double *y, const MKL_INT incy)
{
    if (layout != CblasRowMajor || trans != CblasNoTrans)
    {
        std::fprintf(stderr, "mkl shim: cblas_dgemv only supports row-major no-transpose\n");
        return;
    }
    for (MKL_INT i = 0; i < m; ++i)
    {
        double s = 0.0;
        for (MKL_INT j = 0; j < n; ++j)
            s += a[i * lda + j] * x[j * incx];
        double v = alpha * s;
        if (beta != 0.0)
            v += beta * y[i * incy];
        y[i * incy] = v;
    }
}

struct lpm_shim_sparse_matrix
{
    MKL_INT n;
    long long base;
    const MKL_INT *rs, *re, *ci; /* caller's arrays, as MKL's handle references them */
    const double *v;
    std::vector<double> scratch; /* per-thread partial products of the transposed half */
};

/* The handle references the caller's upper-triangular CSR without copying (as MKL's does). */
sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *A, const sparse_index_base_t indexing, const MKL_INT rows,
                                        const MKL_INT cols, MKL_INT *rows_start, MKL_INT *rows_end,
                                        MKL_INT *col_indx, double *values)
{
    double t0 = now_s();
    if (rows != cols)
        return SPARSE_STATUS_NOT_SUPPORTED;
    auto *M = new lpm_shim_sparse_matrix;
    M->n = rows;
    M->base = (indexing == SPARSE_INDEX_BASE_ONE) ? 1 : 0;
    M->rs = rows_start;
    M->re = rows_end;
    M->ci = col_indx;
    M->v = values;
    *A = M;
    lpm_shim_stats_g.create_seconds += now_s() - t0;
    return SPARSE_STATUS_SUCCESS;
}

/* Threads of the stand-in's own parallel loops.  MKL sizes its thread team by MKL_NUM_THREADS
 * (falling back to the OpenMP setting), independently of the caller's OpenMP loops; the same
 * rule here lets a checker run the reference's own loops on one thread (its assembly scatter
 * races under OpenMP) while the sparse product and the CG vector updates use every core. */
static int shim_threads()
{
    const char *e = std::getenv("MKL_NUM_THREADS");
    const int v = e ? std::atoi(e) : 0;
    if (v > 0)
        return v;
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* y = alpha*A*x + beta*y for A = U + U^T - diag(U) given the upper triangle U (the SYMMETRIC /
 * UPPER descriptor of solver.h:287-289).  Row-parallel gather for U x; the U^T x part is a
 * scatter, accumulated in per-thread buffers and summed afterwards. */
sparse_status_t mkl_sparse_d_mv(const sparse_operation_t operation, const double alpha, const sparse_matrix_t A,
                                const struct matrix_descr descr, const double *x, const double beta, double *y)
{
    (void)operation;
    if (!A)
        return SPARSE_STATUS_NOT_INITIALIZED;
    double t0 = now_s();
    const long long n = A->n, b = A->base;
    const bool sym = descr.type == SPARSE_MATRIX_TYPE_SYMMETRIC;
    const int nt = shim_threads();
    if (sym)
        A->scratch.assign((size_t)nt * n, 0.0);
    double *scr = sym ? A->scratch.data() : nullptr;
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double *yt = sym ? scr + (size_t)t * n : nullptr;
#pragma omp for schedule(static)
        for (long long i = 0; i < n; ++i)
        {
            double s = 0.0;
            const double xi = x[i];
            for (long long p = A->rs[i] - b; p < A->re[i] - b; ++p)
            {
                const long long j = A->ci[p] - b;
                s += A->v[p] * x[j];
                if (sym && j != i)
                    yt[j] += A->v[p] * xi;
            }
            if (sym)
                yt[i] += s;
            else
                y[i] = (beta == 0.0) ? alpha * s : alpha * s + beta * y[i];
        }
        if (sym)
        {
#pragma omp for schedule(static)
            for (long long i = 0; i < n; ++i)
            {
                double s = 0.0;
                for (int q = 0; q < nt; ++q)
                    s += scr[(size_t)q * n + i];
                y[i] = (beta == 0.0) ? alpha * s : alpha * s + beta * y[i];
            }
        }
    }
    lpm_shim_stats_g.spmv_calls++;
    lpm_shim_stats_g.spmv_seconds += now_s() - t0;
    return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_destroy(sparse_matrix_t A)
{
    delete A;
    return SPARSE_STATUS_SUCCESS;
}

/* ---- RCI CG -------------------------------------------------------------------------
 * tmp layout (n x 4): tmp[0:n) = vector to multiply (search direction p), tmp[n:2n) = A*p,
 * tmp[2n:3n) = residual r.  ipar[2] holds the stage of the state machine. */
enum { CG_STAGE_START = 1, CG_STAGE_R0 = 2, CG_STAGE_ITER = 3 };

void dcg_init(const MKL_INT *n, const double *x, const double *b, MKL_INT *rci_request, MKL_INT *ipar,
              double *dpar, double *tmp)
{
    (void)x;
    (void)b;
    for (int i = 0; i < 128; ++i)
    {
        ipar[i] = 0;
        dpar[i] = 0.0;
    }
    ipar[0] = *n;
    ipar[1] = 6;
    ipar[2] = CG_STAGE_START;
    ipar[3] = 0;
    ipar[4] = (*n < 150) ? *n : 150;
    ipar[5] = 1;
    ipar[6] = 1;
    ipar[7] = 1;
    ipar[8] = 0;
    ipar[9] = 1;
    ipar[10] = 0;
    dpar[0] = 1.0e-6;
    dpar[1] = 0.0;
    std::memset(tmp, 0, sizeof(double) * 4 * (size_t)(*n));
    lpm_shim_stats_g.cg_solves++;
    *rci_request = 0;
}

void dcg_check(const MKL_INT *n, const double *x, const double *b, MKL_INT *rci_request, MKL_INT *ipar,
               double *dpar, double *tmp)
{
    (void)x;
    (void)b;
    (void)dpar;
    (void)tmp;
    if (ipar[0] != *n || ipar[4] <= 0)
    {
        *rci_request = -1100;
        return;
    }
    if (lpm_shim_stats_g.cg_maxit_override > 0 && ipar[4] > lpm_shim_stats_g.cg_maxit_override)
        ipar[4] = (MKL_INT)lpm_shim_stats_g.cg_maxit_override;
    if (lpm_shim_stats_g.cg_rtol_override >= 0)
        dpar[0] = lpm_shim_stats_g.cg_rtol_override;
    if (lpm_shim_stats_g.cg_atol_override >= 0)
        dpar[1] = lpm_shim_stats_g.cg_atol_override;
    *rci_request = 0;
}

static double dotv(long long n, const double *a, const double *b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static) num_threads(shim_threads())
    for (long long i = 0; i < n; ++i)
        s += a[i] * b[i];
    return s;
}

void dcg(const MKL_INT *n_, double *x, double *b, MKL_INT *rci_request, MKL_INT *ipar, double *dpar, double *tmp)
{
    double t0 = now_s();
    const long long n = *n_;
    double *p = tmp, *Ap = tmp + n, *r = tmp + 2 * n;
    if (ipar[2] == CG_STAGE_START)
    {
        /* request A*x0 so that r0 = b - A*x0 */
        std::memcpy(p, x, sizeof(double) * n);
        ipar[2] = CG_STAGE_R0;
        *rci_request = 1;
        lpm_shim_stats_g.cg_seconds += now_s() - t0;
        return;
    }
    if (ipar[2] == CG_STAGE_R0)
    {
#pragma omp parallel for schedule(static) num_threads(shim_threads())
        for (long long i = 0; i < n; ++i)
            r[i] = b[i] - Ap[i];
        double rr = dotv(n, r, r);
        dpar[2] = rr;
        dpar[3] = dpar[0] * dpar[2] + dpar[1];
        dpar[4] = rr;
        if (ipar[8] != 0 && dpar[4] <= dpar[3])
        {
            *rci_request = 0;
            lpm_shim_stats_g.cg_seconds += now_s() - t0;
            return;
        }
        std::memcpy(p, r, sizeof(double) * n);
        ipar[2] = CG_STAGE_ITER;
        *rci_request = 1;
        lpm_shim_stats_g.cg_seconds += now_s() - t0;
        return;
    }
    /* CG_STAGE_ITER: Ap holds A*p */
    double pAp = dotv(n, p, Ap);
    if (pAp == 0.0)
    {
        *rci_request = -10;
        lpm_shim_stats_g.cg_failures++;
        lpm_shim_stats_g.cg_seconds += now_s() - t0;
        return;
    }
    const double rr = dpar[4];
    const double alpha = rr / pAp;
#pragma omp parallel for schedule(static) num_threads(shim_threads())
    for (long long i = 0; i < n; ++i)
    {
        x[i] += alpha * p[i];
        r[i] -= alpha * Ap[i];
    }
    ipar[3] += 1;
    lpm_shim_stats_g.cg_iterations++;
    const double rr_new = dotv(n, r, r);
    dpar[5] = dpar[4];
    dpar[4] = rr_new;
    if (ipar[8] != 0 && dpar[4] <= dpar[3])
    {
        *rci_request = 0;
        lpm_shim_stats_g.cg_seconds += now_s() - t0;
        return;
    }
    if (ipar[7] != 0 && ipar[3] >= ipar[4])
    {
        *rci_request = -1;
        lpm_shim_stats_g.cg_failures++;
        lpm_shim_stats_g.cg_seconds += now_s() - t0;
        return;
    }
    const double beta = rr_new / rr;
#pragma omp parallel for schedule(static) num_threads(shim_threads())
    for (long long i = 0; i < n; ++i)
        p[i] = r[i] + beta * p[i];
    *rci_request = 1;
    lpm_shim_stats_g.cg_seconds += now_s() - t0;
}

void dcg_get(const MKL_INT *n, const double *x, const double *b, const MKL_INT *rci_request, const MKL_INT *ipar,
             const double *dpar, const double *tmp, MKL_INT *itercount)
{
    (void)n;
    (void)x;
    (void)b;
    (void)rci_request;
    (void)dpar;
    (void)tmp;
    *itercount = ipar[3];
}

/* PARDISO stand-in: SPD only, solves at phase 33 by a tightly converged CG on the
 * symmetric-upper 1-based CSR (a, ia, ja). */
void PARDISO(void *pt, const MKL_INT *maxfct, const MKL_INT *mnum, const MKL_INT *mtype, const MKL_INT *phase,
             const MKL_INT *n, const void *a, const MKL_INT *ia, const MKL_INT *ja, MKL_INT *perm,
             const MKL_INT *nrhs, MKL_INT *iparm, const MKL_INT *msglvl, void *b, void *x, MKL_INT *error)
{
    (void)pt;
    (void)maxfct;
    (void)mnum;
    (void)perm;
    (void)msglvl;
    *error = 0;
    if (*mtype != 2 || *nrhs != 1)
    {
        *error = -3;
        return;
    }
    if (*phase != 33)
        return;
    iparm[16] = 0;
    sparse_matrix_t A = nullptr;
    mkl_sparse_d_create_csr(&A, SPARSE_INDEX_BASE_ONE, *n, *n, const_cast<MKL_INT *>(ia),
                            const_cast<MKL_INT *>(ia) + 1, const_cast<MKL_INT *>(ja),
                            static_cast<double *>(const_cast<void *>(a)));
    struct matrix_descr d = {SPARSE_MATRIX_TYPE_SYMMETRIC, SPARSE_FILL_MODE_UPPER, SPARSE_DIAG_NON_UNIT};
    const long long nn = *n;
    const double *bb = static_cast<const double *>(b);
    double *xx = static_cast<double *>(x);
    std::vector<double> r(bb, bb + nn), p(bb, bb + nn), q(nn);
    std::fill(xx, xx + nn, 0.0);
    double rr = dotv(nn, r.data(), r.data());
    const double stop = 1e-28 * rr;
    for (long long it = 0; it < 10 * nn && rr > stop; ++it)
    {
        mkl_sparse_d_mv(SPARSE_OPERATION_NON_TRANSPOSE, 1.0, A, d, p.data(), 0.0, q.data());
        double al = rr / dotv(nn, p.data(), q.data());
        for (long long i = 0; i < nn; ++i)
        {
            xx[i] += al * p[i];
            r[i] -= al * q[i];
        }
        double rn = dotv(nn, r.data(), r.data());
        double be = rn / rr;
        rr = rn;
        for (long long i = 0; i < nn; ++i)
            p[i] = r[i] + be * p[i];
    }
    mkl_sparse_destroy(A);
}

void mkl_free_buffers(void) {}
