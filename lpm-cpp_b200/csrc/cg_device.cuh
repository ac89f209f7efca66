// Device helpers shared by the CG kernels (cg.cu: one problem per launch; batch.cu: many
// problems per launch): timed waits, fixed-order warp and block reductions, loads and stores
// with L2 eviction policies, and the sliced-ELL SpMV of one slice.
#pragma once

#include <cstdint>

#include "lpm_internal.cuh"

namespace lpm
{

// one 32-warp block per SM: with <= 64 registers every slice of the 382,500-DOF cube gets its
// own warp (3,985 slices, 4,736 resident warps) and each grid barrier takes 148 arrivals
constexpr int kCGThreads = 1024;
constexpr int kCGMinBlocks = 1;
constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull; // 4 s

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ double wsum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float wsumf(float v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block sum of v (fixed tree: warp butterflies, then warp 0 over the warp totals) into *dst
__device__ __forceinline__ void block_partial_at(double v, double *dst, double *sh)
{
    v = wsum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        sh[w] = v;
    __syncthreads();
    if (w == 0)
    {
        double r = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0.0;
        r = wsum(r);
        if (l == 0)
            *dst = r;
    }
    __syncthreads();
}

// block partial of v into part[blockIdx*2 + slot]
__device__ __forceinline__ void block_partial(double v, double *part, int slot, double *sh)
{
    block_partial_at(v, part + 2 * blockIdx.x + slot, sh);
}

// L2 cache policies: the matrix and its columns are streamed once per iteration (evict-first,
// no L1 allocation, read-only path); the Krylov vectors are gathered many times per iteration
// and must stay in L2 (evict-last on their loads and stores).
__device__ __forceinline__ uint64_t l2_evict_first()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_stream(const double *a, uint64_t pol)
{
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const float *a, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_stream(const int *a, uint64_t pol)
{
    int v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}
// vectors change between phases: volatile keeps these loads where the code puts them
__device__ __forceinline__ double ld_keep(const double *a, uint64_t pol)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ float ld_keep(const float *a, uint64_t pol)
{
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol) : "memory");
    return v;
}
// two consecutive doubles (16-byte aligned) in one load, as ld_keep
__device__ __forceinline__ double2 ld_keep2(const double *a, uint64_t pol)
{
    double2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol) : "memory");
    return v;
}
// two consecutive floats (8-byte aligned) in one load, as ld_keep
__device__ __forceinline__ float2 ld_keep2(const float *a, uint64_t pol)
{
    float2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(a), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ void st_keep2(float *a, float2 v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(a), "f"(v.x), "f"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_keep(double *a, double v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_keep(float *a, float v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}

// q_i = sum_j K_ij (r_j + beta p_old_j) for the row at this lane of slice sl; returns the
// particle id (-1 past the end).  Blocks in ascending connection order, entries row-major.
// U > 1 (callers with registers to spare): U steps of 2 x 2 FP32 blocks in flight at once.
template <typename TK, typename TV, int D, int U = 1>
__device__ __forceinline__ int spmv_slice(int sl, int n, const int *__restrict__ rowptr, const int *__restrict__ perm,
                                          const int64_t *__restrict__ slice_off, const int *__restrict__ col_sell,
                                          const TK *__restrict__ K, const TV *__restrict__ r,
                                          const TV *__restrict__ pold, TV beta, TV acc[D], uint64_t pf,
                                          uint64_t pl, int k0 = 0, int kstep = 1)
{
    // block columns k0, k0 + kstep, ... of the slice (all of them by default)
    constexpr int E = D * D;
    const int lane = threadIdx.x & 31;
    const int pos = sl * kSlice + lane;
    const bool valid = pos < n;
    const int i = valid ? perm[pos] : -1;
    const int myn = valid ? (rowptr[i + 1] - rowptr[i]) : 0;
    const int64_t off = slice_off[sl];
    const int w = (int)(slice_off[sl + 1] - off);
    const int *cp = col_sell + off * kSlice + lane;
    const TK *kp = K + off * E * kSlice + lane;
#pragma unroll
    for (int k = 0; k < D; ++k)
        acc[k] = TV(0);
    if constexpr (U > 1 && sizeof(TK) * E <= 16)
    {
        // Small blocks (2 x 2 FP32: 16 bytes per lane and step): one step moves too little for a
        // warp's chain of column load -> gather to keep HBM busy, so U steps are in flight at
        // once: their columns are fetched one group ahead, then all their gathers and matrix
        // loads are issued before any of them is used.  The sums keep the ascending order.
        int jn[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int kk = k0 + u * kstep;
            jn[u] = (kk < myn) ? ld_stream(cp + (int64_t)kk * kSlice, pf) : 0;
        }
        for (int k = k0; k < w; k += U * kstep)
        {
            int j[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                j[u] = jn[u];
                const int kk = k + (U + u) * kstep;
                jn[u] = (kk < myn) ? ld_stream(cp + (int64_t)kk * kSlice, pf) : 0;
            }
            TV rv[U][D], pv[U][D];
            TK kv[U][E];
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                const int kk = k + u * kstep;
                if (kk < myn)
                {
#pragma unroll
                    for (int c = 0; c < D; ++c)
                    {
                        rv[u][c] = ld_keep(r + (int64_t)j[u] * D + c, pl);
                        pv[u][c] = ld_keep(pold + (int64_t)j[u] * D + c, pl);
                    }
                    const TK *kb = kp + (int64_t)kk * E * kSlice;
#pragma unroll
                    for (int e = 0; e < E; ++e)
                        kv[u][e] = ld_stream(kb + e * kSlice, pf);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                if (k + u * kstep < myn)
                {
                    TV xv[D];
#pragma unroll
                    for (int c = 0; c < D; ++c)
                        xv[c] = rv[u][c] + beta * pv[u][c];
#pragma unroll
                    for (int rr = 0; rr < D; ++rr)
#pragma unroll
                        for (int c = 0; c < D; ++c)
                            acc[rr] += (TV)kv[u][rr * D + c] * xv[c];
                }
            }
        }
        return i;
    }
    // the column of the next step is fetched during this one, so the x gathers never wait on it
    int jn = (myn > k0) ? ld_stream(cp + (int64_t)k0 * kSlice, pf) : 0;
#pragma unroll 2
    for (int k = k0; k < w; k += kstep)
    {
        const int j = jn;
        if (k + kstep < myn)
            jn = ld_stream(cp + (int64_t)(k + kstep) * kSlice, pf);
        if (k < myn)
        {
            TV xv[D];
#pragma unroll
            for (int c = 0; c < D; ++c)
                xv[c] = ld_keep(r + (int64_t)j * D + c, pl) + beta * ld_keep(pold + (int64_t)j * D + c, pl);
            const TK *kb = kp + (int64_t)k * E * kSlice;
            TK kv[E];
#pragma unroll
            for (int e = 0; e < E; ++e)
                kv[e] = ld_stream(kb + e * kSlice, pf);
#pragma unroll
            for (int rr = 0; rr < D; ++rr)
#pragma unroll
                for (int c = 0; c < D; ++c)
                    acc[rr] += (TV)kv[rr * D + c] * xv[c];
        }
    }
    return i;
}

// Maximum warps that share one slice's block columns (the column split below).
constexpr int kMaxColumnSplit = 16;

// Phase A of a CG iteration for the rows of slices [s0, s1), run by the whole block:
// q = K p_new with p_new = r + beta p_old formed on the fly; p_new and q are stored for those
// rows and the thread's share of p_new . q is returned.  With at least one slice per warp each
// warp streams whole slices.  With fewer slices than warps (small problems, or a small share
// of one) S warps share a slice, each taking every S-th block column, so the chain of
// dependent column/gather loads a warp walks is S times shorter; the S partial row sums are
// added in a fixed order through `red` (shared memory, 32 * D * 32 values).  Every thread of
// the block must call it.
template <typename TK, typename TV, int D, int U = 1>
__device__ __forceinline__ double spmv_block(int s0, int s1, int n, const int *__restrict__ rowptr,
                                             const int *__restrict__ perm, const int64_t *__restrict__ slice_off,
                                             const int *__restrict__ col_sell, const TK *__restrict__ K,
                                             const TV *__restrict__ r, const TV *__restrict__ pold,
                                             TV *__restrict__ pnew, TV *__restrict__ q, TV beta, uint64_t pf,
                                             uint64_t pl, TV *red)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int ns = s1 - s0;
    double lpq = 0;
    auto epilogue = [&](int i, const TV *acc) {
        if (i < 0)
            return;
#pragma unroll
        for (int c = 0; c < D; ++c)
        {
            const int64_t k = (int64_t)i * D + c;
            const TV pn = ld_keep(r + k, pl) + beta * ld_keep(pold + k, pl);
            st_keep(pnew + k, pn, pl);
            st_keep(q + k, acc[c], pl);
            lpq += (double)pn * (double)acc[c];
        }
    };
    if (ns <= 0)
        return 0.0;
    if (2 * ns > nw)
    {
        for (int sl = s0 + warp; sl < s1; sl += nw)
        {
            TV acc[D];
            const int i = spmv_slice<TK, TV, D, U>(sl, n, rowptr, perm, slice_off, col_sell, K, r, pold, beta, acc, pf,
                                                   pl);
            epilogue(i, acc);
        }
        return lpq;
    }
    int S = 2;
    while (S < kMaxColumnSplit && ns * S * 2 <= nw)
        S *= 2;
    const int ls = warp / S, part = warp % S;
    TV acc[D];
#pragma unroll
    for (int c = 0; c < D; ++c)
        acc[c] = TV(0);
    int i = -1;
    if (ls < ns)
        i = spmv_slice<TK, TV, D, U>(s0 + ls, n, rowptr, perm, slice_off, col_sell, K, r, pold, beta, acc, pf, pl,
                                     part, S);
    if (ls < ns && part > 0)
#pragma unroll
        for (int c = 0; c < D; ++c)
            red[(warp * D + c) * 32 + lane] = acc[c];
    __syncthreads();
    if (ls < ns && part == 0)
    {
        for (int p = 1; p < S; ++p)
#pragma unroll
            for (int c = 0; c < D; ++c)
                acc[c] += red[((warp + p) * D + c) * 32 + lane];
        epilogue(i, acc);
    }
    __syncthreads();
    return lpq;
}

} // namespace lpm
