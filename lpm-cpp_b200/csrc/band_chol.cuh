// Banded Cholesky factorisation and solves: the numerical core of the direct solver (direct.cu),
// the device counterpart of Solver::LPM_PARDISO (include/solver.h:191-274).
//
// Storage: the lower band of a symmetric positive definite matrix of order n and half-bandwidth
// kd, LAPACK's lower band layout: entry (i, j), j <= i <= j + kd, at AB[(i - j) + j * ldab] with
// ldab >= kd + 1.  Column j of the band is contiguous in i.  The Cholesky factor L overwrites it
// (no fill outside the band).
//
// The factorisation is blocked in column blocks [j0, j0 + jb): the diagonal block is factored,
// the rows below it in the band are solved against it (L21 = A21 L11^-T), and the trailing band
// window is updated (A22 -= L21 L21^T).  Each function below is the whole work of one thread of
// one kernel, and the threads of a kernel never touch one another's outputs, so the kernels are
// race-free and a host loop over the same thread indices computes the same bits.  Every function
// compiles as device and as host code: the tests run this exact code on the CPU.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define LPM_HD __host__ __device__ __forceinline__
#else
#define LPM_HD inline
#endif

namespace lpm
{
namespace band
{

LPM_HD double &at(double *AB, int64_t ldab, int64_t i, int64_t j) { return AB[(i - j) + j * ldab]; }
LPM_HD double at(const double *AB, int64_t ldab, int64_t i, int64_t j) { return AB[(i - j) + j * ldab]; }

// Rows of the band below the block [j0, j0 + jb): [j0 + jb, min(n, j0 + jb + kd)).
LPM_HD int64_t below_end(int64_t n, int64_t kd, int64_t j0, int64_t jb)
{
    const int64_t e = j0 + jb + kd;
    return e < n ? e : n;
}

// One thread: factors the diagonal block in place.  Returns 0, or 1 + the block column whose
// pivot was not positive (the matrix is not positive definite).
LPM_HD int potrf_block(double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb)
{
    for (int64_t jj = 0; jj < jb; ++jj)
    {
        const int64_t j = j0 + jj;
        const double a = at(AB, ldab, j, j);
        if (!(a > 0.0))
            return (int)jj + 1;
        const double d = sqrt(a);
        at(AB, ldab, j, j) = d;
        for (int64_t i = j + 1; i < j0 + jb && i - j <= kd; ++i)
            at(AB, ldab, i, j) = at(AB, ldab, i, j) / d;
        for (int64_t c = j + 1; c < j0 + jb && c - j <= kd; ++c)
        {
            const double lc = at(AB, ldab, c, j);
            for (int64_t i = c; i < j0 + jb && i - j <= kd; ++i)
                at(AB, ldab, i, c) = at(AB, ldab, i, c) - at(AB, ldab, i, j) * lc;
        }
    }
    return 0;
}

// One thread per row i below the block: L(i, j0 .. j0 + jb) = A(i, ..) L11^-T.  Entries outside
// the band (i - j > kd) are zero and stay unstored.
LPM_HD void trsm_row(double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, int64_t i)
{
    for (int64_t jj = 0; jj < jb; ++jj)
    {
        const int64_t j = j0 + jj;
        if (i - j > kd)
            continue;
        double v = at(AB, ldab, i, j);
        for (int64_t k = j0; k < j; ++k)
            if (i - k <= kd)
                v = v - at(AB, ldab, i, k) * at(AB, ldab, j, k);
        at(AB, ldab, i, j) = v / at(AB, ldab, j, j);
    }
}

// One thread per entry (i, c) of the trailing window, c <= i, i - c <= kd:
// A(i, c) -= sum over the block's columns of L(i, j) L(c, j).
LPM_HD void syrk_entry(double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, int64_t i, int64_t c)
{
    double s = 0.0;
    for (int64_t j = j0; j < j0 + jb; ++j)
        if (i - j <= kd)
            s = s + at(AB, ldab, i, j) * at(AB, ldab, c, j);
    at(AB, ldab, i, c) = at(AB, ldab, i, c) - s;
}

// Forward solve L y = b in place, one thread for the block's rows ...
LPM_HD void fwd_block(const double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, double *y)
{
    for (int64_t j = j0; j < j0 + jb; ++j)
    {
        double v = y[j];
        for (int64_t k = j0; k < j; ++k)
            if (j - k <= kd)
                v = v - at(AB, ldab, j, k) * y[k];
        y[j] = v / at(AB, ldab, j, j);
    }
}

// ... then one thread per row i below it: y(i) -= L(i, block) y(block).
LPM_HD void fwd_update_row(const double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, int64_t i, double *y)
{
    double s = 0.0;
    for (int64_t j = j0; j < j0 + jb; ++j)
        if (i - j <= kd)
            s = s + at(AB, ldab, i, j) * y[j];
    y[i] = y[i] - s;
}

// Backward solve L^T x = y in place, blocks from the last: one thread per column j of the block
// takes the finished x below it, y(j) -= sum over rows i below of L(i, j) x(i) ...
LPM_HD void bwd_update_col(const double *AB, int64_t ldab, int64_t kd, int64_t n, int64_t j0, int64_t jb, int64_t j,
                           double *y)
{
    double s = 0.0;
    const int64_t e = below_end(n, kd, j0, jb);
    for (int64_t i = j0 + jb; i < e && i - j <= kd; ++i)
        s = s + at(AB, ldab, i, j) * y[i];
    y[j] = y[j] - s;
}

// ... then one thread solves the block's own triangle, last row first.
LPM_HD void bwd_block(const double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, double *y)
{
    for (int64_t j = j0 + jb - 1; j >= j0; --j)
    {
        double v = y[j];
        for (int64_t k = j + 1; k < j0 + jb; ++k)
            if (k - j <= kd)
                v = v - at(AB, ldab, k, j) * y[k];
        y[j] = v / at(AB, ldab, j, j);
    }
}

} // namespace band
} // namespace lpm
