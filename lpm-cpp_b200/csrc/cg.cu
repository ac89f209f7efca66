// Linear solve of the Newton step: the replacement for Solver::LPM_CG (include/solver.h:277-354),
// i.e. MKL's RCI dcg with mkl_sparse_d_mv on the symmetric upper CSR.
//
// One persistent cooperative launch runs the whole unpreconditioned CG (x0 = 0, stop when
// ||r||^2 <= rtol*||r0||^2 + atol, cap = problem size, the squared-norm test of MKL's dcg with
// dpar[0] = dpar[1] = 1e-12 set at solver.h:312-313).  Per iteration:
//   phase A  q = K p_new, with p_new = r + beta*p_old formed on the fly from the gathered
//            r and p_old (so the direction update needs no pass of its own); partial p.q
//   barrier
//   phase B  x += alpha p_new, r -= alpha q; partial r.r
//   barrier
// Every reduction is a fixed tree, and every block reduces the per-block partials in the same
// order, so all blocks take identical decisions and a run is bit-reproducible.  The grid
// barrier is a sense-counting barrier with a time limit: a wait that exceeds it records
// LPMGPU_ERR_TIMEOUT and the kernel returns.
//
// The SpMV runs on the sliced-ELL layout (lpm_internal.cuh): one thread per particle row, a
// warp per slice of 32 rows.  For block column k every matrix plane load is 256 contiguous
// bytes (cache-streaming: the matrix is read once per iteration) and the x gathers of the 32
// rows hit neighbouring particles, so they coalesce and stay in L2 with the vectors.
//
// Mixed precision (LPMGPU_MIXED): the same kernel on an FP32 copy of K with FP32 Krylov
// vectors (dot products in FP64), inside an FP64 iterative refinement that recomputes the
// true residual b - K x with the FP64 matrix and stops on the same squared-norm rule.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <string>

#include "cg_device.cuh"

namespace lpm
{

struct CGState
{
    int n;              // particle rows
    int nslices;
    int64_t ndof;
    const int *__restrict__ rowptr;     // connection CSR (row lengths)
    const int *__restrict__ perm;       // slice position -> particle
    const int64_t *__restrict__ slice_off;
    const int *__restrict__ col_sell;
    double rtol, atol, abs_stop; // abs_stop >= 0 overrides rtol/atol
    int64_t maxit;
    unsigned *bar;      // [0] arrivals, [1] generation
    double *part;       // [grid][2]
    double *tot;        // [2] reduced totals published by the last block at each barrier
    int64_t *info;      // [0] iterations, [1] status bits (1 maxit, 2 timeout, 4 breakdown), [2..3] rr0/rr bits
    unsigned long long wait_ns; // limit of each grid-barrier wait
};


// Grid barrier fused with the reduction of the per-block partials part[2*b + slot] (used by the
// allocation-free solve below): the last block to arrive sums them (fixed order: thread t takes b = t, t + blockDim, ..., then a fixed
// tree), publishes the total in tot[slot] and releases the others.  Every block returns the
// same total.  Returns false when the wait timed out.
__device__ bool grid_reduce(unsigned *bar, int64_t *info, volatile int *s_fail, const double *part, int slot,
                            double *tot, double *sh, double *out)
{
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        const unsigned gen = ld_acquire(bar + 1);
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        s_last = (arrived == gridDim.x - 1);
        if (!s_last)
        {
            const unsigned long long t0 = gtimer();
            unsigned ns = 32;
            while (ld_acquire(bar + 1) == gen)
            {
                if (gtimer() - t0 > kBarrierTimeoutNs)
                {
                    atomicOr(reinterpret_cast<unsigned long long *>(info + 1), 2ull);
                    *s_fail = 1;
                    break;
                }
                __nanosleep(ns);
                if (ns < 128)
                    ns <<= 1;
            }
            __threadfence();
        }
        else
            __threadfence();
    }
    __syncthreads();
    if (s_last)
    {
        double v = 0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
            v += __ldcg(part + 2 * b + slot);
        v = wsum(v);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0)
            sh[w] = v;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double t = 0;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
                t += sh[q];
            __stcg(tot + slot, t);
            __threadfence();
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        if (*reinterpret_cast<volatile long long *>(info + 1) & 2)
            *s_fail = 1;
        sh[0] = __ldcg(tot + slot);
    }
    __syncthreads();
    *out = sh[0];
    const bool ok = *s_fail == 0;
    __syncthreads();
    return ok;
}

// Grid barrier + all-reduce of the per-block partials part[2*b + slot], with nothing serial on
// the way out: the barrier word only counts arrivals (it starts at zero and is never reset, so
// barrier number e is passed once it reaches (e + 1) * gridDim.x), and after it every block
// sums all partials itself, in one fixed order (thread t takes b = t, t + blockDim, ..., warp
// butterflies, then thread 0 over the warp sums in order), so every block holds the same
// bit-identical total.  The two slots alternate between consecutive reductions, which keeps a
// block that runs one phase ahead from overwriting partials another block is still reading.
// Returns false when the wait timed out (the status word gets bit 2).
__device__ bool grid_allreduce(unsigned *bar, unsigned &epoch, int64_t *info, volatile int *s_fail,
                               const double *part, int slot, double *sh, double *out,
                               unsigned long long wait_ns)
{
    __shared__ double s_tot;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned target = (epoch + 1u) * gridDim.x;
        const unsigned long long t0 = gtimer();
        while ((int)(ld_acquire(bar) - target) < 0)
        {
            if (gtimer() - t0 > wait_ns)
            {
                atomicOr(reinterpret_cast<unsigned long long *>(info + 1), 2ull);
                *s_fail = 1;
                break;
            }
        }
    }
    epoch++;
    __syncthreads();
    if (*s_fail)
        return false;
    double v = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
        v += __ldcg(part + 2 * b + slot);
    v = wsum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
            t += sh[q];
        s_tot = t;
    }
    __syncthreads();
    *out = s_tot;
    return true;
}

template <typename TK, typename TV, int D>
__global__ void __launch_bounds__(kCGThreads, kCGMinBlocks) k_cg(CGState s, const TK *__restrict__ K, const TV *__restrict__ b,
                                                   TV *__restrict__ x, TV *__restrict__ r, TV *__restrict__ pa,
                                                   TV *__restrict__ pb, TV *__restrict__ q)
{
    __shared__ double sh[32];
    __shared__ int s_fail;
    __shared__ TV red[32 * D * 32];
    if (threadIdx.x == 0)
        s_fail = 0;
    __syncthreads();
    unsigned epoch = 0;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // each block owns a contiguous, equal share of the slices (balanced, neighbours share L1)
    const int s0 = (int)((int64_t)blockIdx.x * s.nslices / gridDim.x);
    const int s1 = (int)((int64_t)(blockIdx.x + 1) * s.nslices / gridDim.x);
    const int warp = threadIdx.x >> 5;
    const uint64_t pf = l2_evict_first(), pl = l2_evict_last();

    double loc = 0;
    for (int64_t k = gt; k < s.ndof; k += T)
    {
        const TV v = b[k];
        st_keep(r + k, v, pl);
        st_keep(x + k, TV(0), pl);
        st_keep(pa + k, TV(0), pl);
        loc += (double)v * (double)v;
    }
    block_partial(loc, s.part, 0, sh);
    double rr;
    if (!grid_allreduce(s.bar, epoch, s.info, &s_fail, s.part, 0, sh, &rr, s.wait_ns))
        return;
    const double stop = (s.abs_stop >= 0) ? s.abs_stop : s.rtol * rr + s.atol;
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        s.info[0] = 0;
        reinterpret_cast<double *>(s.info)[2] = rr;
        reinterpret_cast<double *>(s.info)[3] = rr;
    }
    if (rr <= stop)
        return;
    TV beta = TV(0);
    TV *pold = pa, *pnew = pb;
    for (int64_t it = 1;; ++it)
    {
        const double lpq = spmv_block<TK, TV, D>(s0, s1, s.n, s.rowptr, s.perm, s.slice_off, s.col_sell, K, r,
                                                   pold, pnew, q, beta, pf, pl, red);
        block_partial(lpq, s.part, 1, sh);
        double pq;
        if (!grid_allreduce(s.bar, epoch, s.info, &s_fail, s.part, 1, sh, &pq, s.wait_ns))
            return;
        if (pq == 0.0)
        {
            if (blockIdx.x == 0 && threadIdx.x == 0)
            {
                s.info[0] = it - 1;
                atomicOr(reinterpret_cast<unsigned long long *>(s.info + 1), 4ull);
            }
            return;
        }
        const double alpha = rr / pq;
        const TV al = (TV)alpha;
        double lrr = 0;
        for (int64_t k = gt; k < s.ndof; k += T)
        {
            const TV pn = ld_keep(pnew + k, pl);
            st_keep(x + k, ld_keep(x + k, pl) + al * pn, pl);
            const TV rv = ld_keep(r + k, pl) - al * ld_keep(q + k, pl);
            st_keep(r + k, rv, pl);
            lrr += (double)rv * (double)rv;
        }
        block_partial(lrr, s.part, 0, sh);
        double rn;
        if (!grid_allreduce(s.bar, epoch, s.info, &s_fail, s.part, 0, sh, &rn, s.wait_ns))
            return;
        const bool done = rn <= stop;
        const bool capped = it >= s.maxit;
        if (done || capped)
        {
            if (blockIdx.x == 0 && threadIdx.x == 0)
            {
                s.info[0] = it;
                reinterpret_cast<double *>(s.info)[3] = rn;
                if (!done)
                    atomicOr(reinterpret_cast<unsigned long long *>(s.info + 1), 1ull);
            }
            return;
        }
        beta = (TV)(rn / rr);
        rr = rn;
        TV *t = pold;
        pold = pnew;
        pnew = t;
    }
}

// ---- helpers for the mixed-precision refinement
template <typename TA, typename TB>
__global__ void k_convert(int64_t m, const TA *__restrict__ a, TB *__restrict__ b)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        b[k] = (TB)a[k];
}

__global__ void k_add_f32(int64_t m, const float *__restrict__ d, double *__restrict__ x)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        x[k] += (double)d[k];
}

// r = b - K x (FP64), partial ||r||^2 per block
template <int D>
__global__ void __launch_bounds__(256) k_residual64(int n, int nslices, const int *__restrict__ rowptr,
                                                    const int *__restrict__ perm, const int64_t *__restrict__ slice_off,
                                                    const int *__restrict__ col_sell, const double *__restrict__ K,
                                                    const double *__restrict__ b, const double *__restrict__ x,
                                                    double *__restrict__ r, double *__restrict__ part)
{
    __shared__ double sh[32];
    const int W = (gridDim.x * blockDim.x) >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    double loc = 0;
    for (int sl = gw; sl < nslices; sl += W)
    {
        double acc[D];
        const int i = spmv_slice<double, double, D>(sl, n, rowptr, perm, slice_off, col_sell, K, x, x, 0.0, acc,
                                                    l2_evict_first(), l2_evict_last());
        if (i >= 0)
            for (int c = 0; c < D; ++c)
            {
                const int64_t k = (int64_t)i * D + c;
                const double v = b[k] - acc[c];
                r[k] = v;
                loc += v * v;
            }
    }
    block_partial(loc, part, 0, sh);
}

__global__ void k_sum_partials(int nblk, const double *__restrict__ part, double *__restrict__ out)
{
    __shared__ double sh[32];
    double v = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        v += part[2 * b];
    v = wsum(v);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        double t = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : 0.0;
        t = wsum(t);
        if (threadIdx.x == 0)
            *out = t;
    }
}

// The default CG grid: one block per SM (kCGMinBlocks per SM when they fit), at most one block per
// slice.  Every grid up to it is co-resident, as the cooperative launch needs.
template <typename TK, typename TV, int D>
static cudaError_t cg_grid_rule(const Problem &p, int *grid_out)
{
    static int occ_cache[2][2][4] = {};
    int &occ = occ_cache[sizeof(TK) == 8][sizeof(TV) == 8][D];
    if (occ == 0)
    {
        const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg<TK, TV, D>, kCGThreads, 0);
        if (e != cudaSuccess)
            return e;
        if (occ < 1)
            occ = 1;
    }
    int grid = p.num_sms * std::min(occ, kCGMinBlocks);
    if (grid > p.nslices)
        grid = std::max(1, p.nslices);
    if (grid > kMaxGridBlocks)
        grid = kMaxGridBlocks;
    *grid_out = grid;
    return cudaSuccess;
}

template <typename TK, typename TV, int D>
static cudaError_t run_cg(Problem &p, const TK *K, const TV *b, TV *x, TV *r, TV *pa, TV *pb, TV *q, double rtol,
                          double atol, double abs_stop, int64_t maxit, CGResult &out, double *rr_final)
{
    cudaError_t e;
    int grid = 0;
    if ((e = cg_grid_rule<TK, TV, D>(p, &grid)) != cudaSuccess)
        return e;
    if (p.cg_grid > 0 && p.cg_grid < grid)
        grid = p.cg_grid; // a tuned grid only ever lowers the default, so it stays co-resident
    CGState s;
    s.n = p.n;
    s.nslices = p.nslices;
    s.ndof = (int64_t)p.n * D;
    s.rowptr = p.cstart;
    s.perm = p.perm;
    s.slice_off = p.slice_off;
    s.col_sell = p.col_sell;
    s.rtol = rtol;
    s.atol = atol;
    s.abs_stop = abs_stop;
    s.maxit = maxit;
    s.bar = p.barrier;
    s.part = p.partials;
    s.tot = p.partials + 2 * kMaxGridBlocks;
    s.info = p.cg_info;
    s.wait_ns = p.wait_ns;
    if ((e = cudaMemsetAsync(p.barrier, 0, 2 * sizeof(unsigned), p.stream)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(p.cg_info, 0, 4 * sizeof(int64_t), p.stream)) != cudaSuccess)
        return e;
    void *args[] = {&s, &K, &b, &x, &r, &pa, &pb, &q};
    if ((e = cudaEventRecord(p.cg_ev[0], p.stream)) != cudaSuccess)
        return e;
    e = cudaLaunchCooperativeKernel((const void *)k_cg<TK, TV, D>, dim3(grid), dim3(kCGThreads), args, 0, p.stream);
    if (e != cudaSuccess)
        return e;
    if ((e = cudaEventRecord(p.cg_ev[1], p.stream)) != cudaSuccess)
        return e;
    p.ctr.kernel_launches++;
    p.ctr.cg_launches++;
    if ((e = cudaMemcpyAsync(p.cg_info_host, p.cg_info, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, p.stream)) !=
        cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(p.stream)) != cudaSuccess)
        return e;
    out.iters += p.cg_info_host[0];
    p.ctr.cg_iters += p.cg_info_host[0];
    {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.cg_ev[0], p.cg_ev[1]) == cudaSuccess)
            p.ctr.cg_kernel_seconds += ms * 1e-3;
        static const bool log = std::getenv("LPMGPU_LOG") != nullptr;
        if (log)
            std::fprintf(stderr, "lpmgpu cg launch %lld: %s%s iters=%lld ms=%.3f grid=%d\n",
                         (long long)p.ctr.cg_launches, sizeof(TK) == 8 ? "fp64" : "fp32", D == 2 ? "/2d" : "/3d",
                         (long long)p.cg_info_host[0], ms, grid);
    }
    if (p.cg_info_host[1] & 1)
        out.maxit_hits++;
    if (p.cg_info_host[1] & 2)
        out.timeout = true;
    if (p.cg_info_host[1] & 4)
        out.breakdown = true;
    if (rr_final)
        *rr_final = reinterpret_cast<double *>(p.cg_info_host)[3];
    return cudaSuccess;
}

template <int D>
static cudaError_t solve_dim(Problem &p, CGResult &out)
{
    const int64_t ndof = (int64_t)p.n * D;
    const int64_t maxit = p.desc.cg_maxit > 0 ? p.desc.cg_maxit : ndof;
    if (p.desc.precision != LPMGPU_MIXED)
        return run_cg<double, double, D>(p, p.K, p.res, p.x, p.r, p.p0, p.p1, p.q, p.desc.cg_rtol, p.desc.cg_atol,
                                         -1.0, maxit, out, nullptr);
    // FP32 Krylov solve inside FP64 iterative refinement on the same stopping rule
    cudaError_t e;
    // rr0 = ||b||^2 via r = b - K*0
    if ((e = cudaMemsetAsync(p.x, 0, sizeof(double) * ndof, p.stream)) != cudaSuccess)
        return e;
    auto true_residual = [&](double &val) -> cudaError_t {
        cudaError_t e2 = enqueue_true_residual(p);
        if (e2 == cudaSuccess)
            e2 = cudaStreamSynchronize(p.stream);
        val = true_residual_result(p);
        return e2;
    };
    double rr0 = 0, rr = 0;
    if ((e = true_residual(rr0)) != cudaSuccess)
        return e;
    const double stop = p.desc.cg_rtol * rr0 + p.desc.cg_atol;
    rr = rr0;
    for (int ref = 0; ref < 30 && !(rr <= stop); ++ref)
    {
        if ((e = enqueue_r_to_b32(p)) != cudaSuccess)
            return e;
        // the inner solve aims a little below the outer target, measured on its own residual
        CGResult inner;
        double rr_in = 0;
        if ((e = run_cg<float, float, D>(p, p.K32, p.b32, p.x32, p.r32, p.pa32, p.pb32, p.q32, 0.0, 0.0, 0.25 * stop,
                                         maxit, inner, &rr_in)) != cudaSuccess)
            return e;
        out.iters += inner.iters;
        out.maxit_hits += inner.maxit_hits;
        out.timeout = out.timeout || inner.timeout;
        out.breakdown = out.breakdown || inner.breakdown;
        out.refinements++;
        if (inner.timeout)
            break;
        if ((e = enqueue_add_x32(p)) != cudaSuccess)
            return e;
        if ((e = true_residual(rr)) != cudaSuccess)
            return e;
        if (inner.iters == 0)
            break;
    }
    return cudaSuccess;
}

// r = b - K x (FP64 matrix) and ||r||^2 -> the pinned slot read by true_residual_result
cudaError_t enqueue_true_residual(Problem &p)
{
    const int64_t ndof = (int64_t)p.n * p.dim;
    const int nb_res = std::min(div_up(ndof, 256), 4 * p.num_sms);
    double *dst = reinterpret_cast<double *>(p.cg_info) + 5;
    if (p.dim == 2)
        k_residual64<2><<<nb_res, 256, 0, p.stream>>>(p.n, p.nslices, p.cstart, p.perm, p.slice_off, p.col_sell, p.K,
                                                      p.res, p.x, p.r, p.partials);
    else
        k_residual64<3><<<nb_res, 256, 0, p.stream>>>(p.n, p.nslices, p.cstart, p.perm, p.slice_off, p.col_sell, p.K,
                                                      p.res, p.x, p.r, p.partials);
    k_sum_partials<<<1, 256, 0, p.stream>>>(nb_res, p.partials, dst);
    p.ctr.kernel_launches += 2;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    return cudaMemcpyAsync(p.cg_info_host + 5, dst, sizeof(double), cudaMemcpyDeviceToHost, p.stream);
}

double true_residual_result(const Problem &p)
{
    return reinterpret_cast<const double *>(p.cg_info_host)[5];
}

cudaError_t enqueue_r_to_b32(Problem &p)
{
    const int64_t ndof = (int64_t)p.n * p.dim;
    k_convert<double, float><<<std::min(div_up(ndof, 256), 8 * p.num_sms), 256, 0, p.stream>>>(ndof, p.r, p.b32);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

cudaError_t enqueue_res_to_b32(Problem &p)
{
    const int64_t ndof = (int64_t)p.n * p.dim;
    k_convert<double, float><<<std::min(div_up(ndof, 256), 8 * p.num_sms), 256, 0, p.stream>>>(ndof, p.res, p.b32);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

cudaError_t enqueue_add_x32(Problem &p)
{
    const int64_t ndof = (int64_t)p.n * p.dim;
    k_add_f32<<<std::min(div_up(ndof, 256), 8 * p.num_sms), 256, 0, p.stream>>>(ndof, p.x32, p.x);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

__global__ void k_to_f32(int64_t m, const double *__restrict__ a, float *__restrict__ b)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        b[k] = (float)a[k];
}

cudaError_t launch_k_to_f32(Problem &p)
{
    const int64_t m = p.nsb * p.dim * p.dim * kSlice;
    k_to_f32<<<std::min(div_up(m, 256), 16 * p.num_sms), 256, 0, p.stream>>>(m, p.K, p.K32);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

cudaError_t solve_linear(Problem &p, CGResult &out)
{
    return p.dim == 2 ? solve_dim<2>(p, out) : solve_dim<3>(p, out);
}

// ---- autotuner of the CG launch shape (no counterpart in the reference)
//
// The persistent CG kernel's cost per iteration is the matrix stream plus two grid barriers.  On
// large problems every SM streams and the default grid (one block per SM) is best; on small ones
// the barriers dominate and fewer, fuller blocks can be faster.  The tuner times `iterations` CG
// iterations of this problem's own matrix for each candidate grid (the default and its 3/4, 1/2,
// 1/4, 1/8, 1/16), twice each, and keeps the fastest by its second timing.  Candidates are never
// above the default, so every one is co-resident.
template <typename TK, typename TV, int D>
static cudaError_t tune_dim(Problem &p, int iterations, lpmgpu_tune_result *res, const TK *K, const TV *b, TV *x,
                            TV *r, TV *pa, TV *pb, TV *q)
{
    int g0 = 0;
    cudaError_t e = cg_grid_rule<TK, TV, D>(p, &g0);
    if (e != cudaSuccess)
        return e;
    std::vector<int> cand;
    for (int f : {16, 12, 8, 4, 2, 1}) // 16/16, 12/16, ... of the default
    {
        const int g = std::max(1, g0 * f / 16);
        if (std::find(cand.begin(), cand.end(), g) == cand.end() && (int)cand.size() < LPMGPU_TUNE_MAX)
            cand.push_back(g);
    }
    const int saved = p.cg_grid;
    const lpmgpu_counters ctr = p.ctr;
    int best = g0;
    double best_us = 0;
    res->ncandidates = (int32_t)cand.size();
    for (size_t k = 0; k < cand.size(); ++k)
    {
        p.cg_grid = cand[k];
        double us = 0;
        for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep)
        {
            CGResult cr;
            e = run_cg<TK, TV, D>(p, K, b, x, r, pa, pb, q, 0.0, 0.0, 0.0, iterations, cr, nullptr);
            float ms = 0;
            if (e == cudaSuccess && (e = cudaEventElapsedTime(&ms, p.cg_ev[0], p.cg_ev[1])) == cudaSuccess)
                us = cr.iters > 0 ? 1e3 * ms / (double)cr.iters : 0.0;
            if (cr.timeout)
            {
                set_last_error("a device-side barrier wait timed out while tuning the CG kernel");
                e = cudaErrorLaunchTimeout;
            }
        }
        if (e != cudaSuccess)
            break;
        res->grid[k] = cand[k];
        res->us_per_iter[k] = us;
        if (us > 0 && (best_us == 0 || us < best_us))
        {
            best_us = us;
            best = cand[k];
        }
    }
    p.ctr = ctr; // tuning launches do not count as solves
    p.cg_grid = (e == cudaSuccess) ? (best == g0 ? 0 : best) : saved;
    res->grid_default = g0;
    res->grid_chosen = best;
    return e;
}

} // namespace lpm

extern "C" {

int32_t lpmgpu_set_cg_grid(lpmgpu_solver *h, int32_t grid)
{
    if (!h || grid < 0)
        return LPMGPU_ERR_INVALID_ARG;
    h->p.cg_grid = grid;
    return LPMGPU_OK;
}

int32_t lpmgpu_set_wait_limit_ns(lpmgpu_solver *h, int64_t ns)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    h->p.wait_ns = ns > 0 ? (unsigned long long)ns : lpm::kBarrierTimeoutNs;
    return LPMGPU_OK;
}

int32_t lpmgpu_autotune(lpmgpu_solver *h, int32_t iterations, lpmgpu_tune_result *out)
{
    using namespace lpm;
    if (!h || !out || iterations < 1 || iterations > 100000)
        return LPMGPU_ERR_INVALID_ARG;
    *out = lpmgpu_tune_result{};
    Problem &p = h->p;
    cudaError_t e = cudaSetDevice(p.device);
    // K from the current state, as the next load step assembles it; the right-hand side is the
    // diagonal before the BC elimination, which is nonzero for every row
    if (e == cudaSuccess)
        e = enqueue_assemble(p, true);
    const int64_t ndof = (int64_t)p.n * p.dim;
    if (e == cudaSuccess && p.desc.precision == LPMGPU_MIXED)
    {
        k_convert<double, float><<<std::min(div_up(ndof, 256), 8 * p.num_sms), 256, 0, p.stream>>>(ndof, p.diag_raw,
                                                                                                   p.b32);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
    {
        out->precision = p.desc.precision;
        if (p.desc.precision == LPMGPU_MIXED)
            e = p.dim == 2 ? tune_dim<float, float, 2>(p, iterations, out, p.K32, p.b32, p.x32, p.r32, p.pa32, p.pb32,
                                                       p.q32)
                           : tune_dim<float, float, 3>(p, iterations, out, p.K32, p.b32, p.x32, p.r32, p.pa32, p.pb32,
                                                       p.q32);
        else
            e = p.dim == 2 ? tune_dim<double, double, 2>(p, iterations, out, p.K, p.diag_raw, p.x, p.r, p.p0, p.p1, p.q)
                           : tune_dim<double, double, 3>(p, iterations, out, p.K, p.diag_raw, p.x, p.r, p.p0, p.p1, p.q);
    }
    if (e == cudaErrorLaunchTimeout)
        return LPMGPU_ERR_TIMEOUT;
    if (e != cudaSuccess)
    {
        set_last_error(std::string("lpmgpu_autotune: ") + cudaGetErrorString(e));
        return LPMGPU_ERR_CUDA;
    }
    return LPMGPU_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------------------
// Allocation-free CG on a caller-supplied block-CSR matrix.
//
// Some callers cannot allocate device memory.  A plugin that runs inside a host program which
// owns all device memory through its own pool or arena may not call cudaMalloc behind that
// allocator's back, and a latency-bound loop cannot afford cudaMalloc/cudaFree, which may
// synchronise the whole device.  For them the solve below takes every input and output from
// the caller and keeps its own work vectors, reduction partials and barrier words in the
// file-scope array g_noalloc_scratch, which every GPU that loads this library holds (about
// 8 MiB) until the process exits.
//
// Limits and caveats:
//  * at most kNoAllocMaxDof unknowns (rows * dim); larger systems are rejected;
//  * all calls on a device share the one array and it keeps the last call's contents, so
//    calls that overlap on the GPU (two streams, two host threads) race; serialise them;
//  * the first call on a device looks up the array's device address (set-up) and should
//    come before any stream capture begins; a cudaDeviceReset of that device invalidates the
//    looked-up address, so the entry point must not be used after one;
//  * the call waits for its stream before returning, and reports a solve that reached its
//    iteration cap (LPMGPU_ERR_CG_MAXIT) or broke down with p.Ap == 0 (LPMGPU_ERR_CG_BREAKDOWN).
namespace lpm
{

constexpr int64_t kNoAllocMaxDof = int64_t(1) << 18; // 262,144 unknowns
constexpr int kNoAllocMaxBlocks = 1024;
// r, p_a, p_b, q | per-block partials [2*blocks] | totals [2] | status words [4] | barrier [2]
constexpr int64_t kNoAllocDoubles = 4 * kNoAllocMaxDof + 2 * kNoAllocMaxBlocks + 2 + 4 + 2;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

struct CGBsr
{
    int nrows;
    int64_t ndof;
    const int *__restrict__ rowptr;
    const int *__restrict__ col;
    const double *__restrict__ val; // row-major d x d blocks
    double rtol, atol;
    int64_t maxit;
    unsigned *bar;
    double *part;
    double *tot;
    int64_t *info;
};

template <int D>
__global__ void __launch_bounds__(kCGThreads, kCGMinBlocks)
    k_cg_bsr_noalloc(CGBsr s, const double *__restrict__ b, double *__restrict__ x, double *__restrict__ r,
                     double *__restrict__ pa, double *__restrict__ pb, double *__restrict__ q)
{
    constexpr int E = D * D;
    __shared__ double sh[32];
    __shared__ int s_fail;
    if (threadIdx.x == 0)
        s_fail = 0;
    __syncthreads();
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double loc = 0;
    for (int64_t k = gt; k < s.ndof; k += T)
    {
        const double v = b[k];
        r[k] = v;
        x[k] = 0.0;
        pa[k] = 0.0;
        loc += v * v;
    }
    block_partial(loc, s.part, 0, sh);
    double rr;
    if (!grid_reduce(s.bar, s.info, &s_fail, s.part, 0, s.tot, sh, &rr))
        return;
    const double stop = s.rtol * rr + s.atol;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        s.info[0] = 0;
    if (rr <= stop)
        return;
    double beta = 0.0;
    double *pold = pa, *pnew = pb;
    for (int64_t it = 1;; ++it)
    {
        double lpq = 0;
        for (int64_t row = gt; row < s.nrows; row += T)
        {
            double acc[D];
#pragma unroll
            for (int c = 0; c < D; ++c)
                acc[c] = 0.0;
            for (int bk = s.rowptr[row]; bk < s.rowptr[row + 1]; ++bk)
            {
                const int64_t j = s.col[bk];
                double xv[D];
#pragma unroll
                for (int c = 0; c < D; ++c)
                    xv[c] = r[j * D + c] + beta * pold[j * D + c];
                const double *v = s.val + (int64_t)bk * E;
#pragma unroll
                for (int rr2 = 0; rr2 < D; ++rr2)
#pragma unroll
                    for (int c = 0; c < D; ++c)
                        acc[rr2] += v[rr2 * D + c] * xv[c];
            }
#pragma unroll
            for (int c = 0; c < D; ++c)
            {
                const int64_t k = row * D + c;
                const double pn = r[k] + beta * pold[k];
                pnew[k] = pn;
                q[k] = acc[c];
                lpq += pn * acc[c];
            }
        }
        block_partial(lpq, s.part, 1, sh);
        double pq;
        if (!grid_reduce(s.bar, s.info, &s_fail, s.part, 1, s.tot, sh, &pq))
            return;
        if (pq == 0.0)
        {
            if (blockIdx.x == 0 && threadIdx.x == 0)
            {
                s.info[0] = it - 1;
                atomicOr(reinterpret_cast<unsigned long long *>(s.info + 1), 4ull);
            }
            return;
        }
        const double alpha = rr / pq;
        double lrr = 0;
        for (int64_t k = gt; k < s.ndof; k += T)
        {
            x[k] = x[k] + alpha * pnew[k];
            const double rv = r[k] - alpha * q[k];
            r[k] = rv;
            lrr += rv * rv;
        }
        block_partial(lrr, s.part, 0, sh);
        double rn;
        if (!grid_reduce(s.bar, s.info, &s_fail, s.part, 0, s.tot, sh, &rn))
            return;
        if (rn <= stop || it >= s.maxit)
        {
            if (blockIdx.x == 0 && threadIdx.x == 0)
            {
                s.info[0] = it;
                if (!(rn <= stop))
                    atomicOr(reinterpret_cast<unsigned long long *>(s.info + 1), 1ull);
            }
            return;
        }
        beta = rn / rr;
        rr = rn;
        double *t = pold;
        pold = pnew;
        pnew = t;
    }
}

// The device address of the array in the current device's context, looked up on every call (the
// lookup allocates nothing): a cached address would dangle after the host application resets the
// device or re-creates its context, which reloads the module.
static cudaError_t noalloc_scratch(int dev, double **out)
{
    if (dev < 0)
        return cudaErrorInvalidDevice;
    double *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
        return e;
    *out = ptr;
    return cudaSuccess;
}

template <int D>
static cudaError_t noalloc_launch(double *scr, int grid, const CGBsr &s0, const double *b, double *x,
                                  cudaStream_t stream, int64_t *status)
{
    CGBsr s = s0;
    double *r = scr, *pa = scr + kNoAllocMaxDof, *pb = scr + 2 * kNoAllocMaxDof, *q = scr + 3 * kNoAllocMaxDof;
    s.part = scr + 4 * kNoAllocMaxDof;
    s.tot = s.part + 2 * kNoAllocMaxBlocks;
    s.info = reinterpret_cast<int64_t *>(s.tot + 2);
    s.bar = reinterpret_cast<unsigned *>(s.tot + 6);
    // the barrier words and status must start at zero; the vectors are written before use
    cudaError_t e = cudaMemsetAsync(s.info, 0, 4 * sizeof(int64_t) + 2 * sizeof(double), stream);
    if (e != cudaSuccess)
        return e;
    void *args[] = {&s, &b, &x, &r, &pa, &pb, &q};
    e = cudaLaunchCooperativeKernel((const void *)k_cg_bsr_noalloc<D>, dim3(grid), dim3(kCGThreads), args, 0, stream);
    if (e != cudaSuccess)
        return e;
    e = cudaMemcpyAsync(status, s.info, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess)
        return e;
    return cudaStreamSynchronize(stream);
}

} // namespace lpm

extern "C" int32_t lpmgpu_cg_bsr_noalloc(int32_t dim, int32_t nrows, const int32_t *rowptr, const int32_t *colidx,
                                         const double *values, const double *b, double *x, double rtol, double atol,
                                         int64_t maxit, void *stream, int64_t *iterations)
{
    using namespace lpm;
    if ((dim != 2 && dim != 3) || nrows <= 0 || !rowptr || !colidx || !values || !b || !x)
        return LPMGPU_ERR_INVALID_ARG;
    if ((int64_t)nrows * dim > kNoAllocMaxDof)
    {
        set_last_error("lpmgpu_cg_bsr_noalloc: more than 262144 unknowns (the size of its static scratch)");
        return LPMGPU_ERR_INVALID_ARG;
    }
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    double *scr = nullptr;
    if (e == cudaSuccess)
        e = noalloc_scratch(dev, &scr);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = (dim == 2) ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg_bsr_noalloc<2>, kCGThreads, 0)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg_bsr_noalloc<3>, kCGThreads, 0);
    if (e != cudaSuccess)
    {
        set_last_error(std::string("lpmgpu_cg_bsr_noalloc: ") + cudaGetErrorString(e));
        return e == cudaErrorNoDevice ? LPMGPU_ERR_NO_DEVICE : LPMGPU_ERR_CUDA;
    }
    int grid = sms * std::max(1, std::min(occ, kCGMinBlocks));
    grid = std::min(grid, kNoAllocMaxBlocks);
    grid = (int)std::min<int64_t>(grid, (nrows + kCGThreads - 1) / kCGThreads);
    grid = std::max(grid, 1);
    CGBsr s{};
    s.nrows = nrows;
    s.ndof = (int64_t)nrows * dim;
    s.rowptr = rowptr;
    s.col = colidx;
    s.val = values;
    s.rtol = rtol;
    s.atol = atol;
    s.maxit = maxit > 0 ? maxit : s.ndof;
    int64_t status[2] = {0, 0};
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    e = (dim == 2) ? noalloc_launch<2>(scr, grid, s, b, x, st, status) : noalloc_launch<3>(scr, grid, s, b, x, st, status);
    if (e != cudaSuccess)
    {
        set_last_error(std::string("lpmgpu_cg_bsr_noalloc: ") + cudaGetErrorString(e));
        return LPMGPU_ERR_CUDA;
    }
    if (iterations)
        *iterations = status[0];
    // status bits of k_cg_bsr_noalloc: 2 a barrier wait timed out, 4 p.Ap == 0, 1 cap reached
    if (status[1] & 2)
    {
        set_last_error("lpmgpu_cg_bsr_noalloc: a device-side barrier wait timed out");
        return LPMGPU_ERR_TIMEOUT;
    }
    if (status[1] & 4)
    {
        set_last_error("lpmgpu_cg_bsr_noalloc: CG broke down (p.Ap == 0: the matrix is singular or indefinite)");
        return LPMGPU_ERR_CG_BREAKDOWN;
    }
    if (status[1] & 1)
    {
        set_last_error("lpmgpu_cg_bsr_noalloc: CG reached its iteration cap without meeting the tolerance");
        return LPMGPU_ERR_CG_MAXIT;
    }
    return LPMGPU_OK;
}
