// Many independent problems on one GPU: the batched persistent CG and the runtime that advances
// every problem's load path in rounds.
//
// Batched CG.  One cooperative launch solves the Newton systems of many problems (any mix of
// 2D and 3D, each with its own sliced-ELL matrix and Krylov vectors), each with its own
// stopping test, iteration cap and scalars: the unpreconditioned CG of Solver::LPM_CG
// (include/solver.h:277-354, MKL RCI dcg on the squared-norm test) per problem.
//   * The split: the active problems' matrix costs are laid end to end and cut into one equal
//     segment per physical block (one block per SM); a problem's piece in a block is its part of
//     that segment in whole slices (SpMV phase) and, in proportion, of its unknowns (update
//     phase).  Small problems share a block, large ones span many; every SM carries the same
//     matrix volume whatever the mix.
//   * Each piece writes one partial per reduction.  After the counting grid barrier every block
//     sums each problem's partials in the same fixed order (32-wide warp sums in piece order),
//     takes the same per-problem decisions (alpha; converged, capped or broken down; the mixed
//     solves' refinement steps) and, when problems leave, re-splits the GPU over the rest, so
//     the tail of a batch runs on the whole GPU.
//   * Mixed members run their FP64 refinement inside the launch: x64 += x32, the true FP64
//     residual and the restart of the next inner FP32 solve, while the others keep iterating.
//   * All waits are bounded (4 s); a timeout sets a flag and every block returns.
//
// Runtime.  Each member follows SolverStatic::solveProblem / solveProblemStep
// (include/solver_static.h:65-152) exactly as lpmgpu_solve_load_step does: apply the load
// step, assemble, modified Newton with K fixed, J2 state + static damage, the damage loop, and
// on Newton failure reset + halve + run both halves.  A round issues every member's next piece
// of device work on the member's stream, one batched CG for all members that need a linear
// solve, and then waits once for all of them before the host takes the members' decisions.
// Also the nonlocal damage and elastic-damage particles, through the same per-member kernels,
// and fatigue members (lpmgpu_batch_add_fatigue): SolverFatigue's static steps and cycles
// (include/solver_fatigue.h:221-302), whose steps go through the same rounds.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "bulk_copy.cuh"
#include "cg_device.cuh"

namespace lpm
{

constexpr int kMaxBatch = 256;                       // problems in one launch (their CG scalars live in
                                                     // every block's shared memory)
constexpr int kMaxVirt = kMaxGridBlocks + kMaxBatch; // virtual blocks
constexpr int kMaxStage = 1024 + kMaxBatch;          // virtual blocks a launch may use (grid <= 1024)
constexpr int kMaxMembers = 4096;                    // running members of one batch (launched in groups
                                                     // of at most kMaxBatch)
constexpr int kDefaultLanes = 1;                     // lanes of a new batch (LPMGPU_BATCH_LANES overrides)
constexpr int64_t kDefaultSoloBytes = 192000000;      // per-iteration matrix stream of a solo member

struct BInst
{
    int dim, n, nslices;
    int fresh;          // 1: the solve starts here (r = b, x = 0); 0: it resumes a paused solve
    int refine;         // 1: FP32 inner solves inside an FP64 iterative refinement run in this launch
    int pad;
    int64_t ndof, cost; // cost: block slots x (d^2 + 1) (matrix entries + column index), the split weight
    const int *rowptr, *perm;
    const int64_t *slice_off;
    const int *col_sell;
    const void *K, *b;
    void *x, *r, *pa, *pb, *q;
    // the single-reduction inner solves (k_cg_batch_sr): second buffers of r, w = A r (first: q)
    // and s = A p (first: pb); p is pa
    void *r1, *w1, *s1;
    double rtol, atol, abs_stop;
    int64_t maxit;
    // refinement (refine = 1): the FP64 system K64 x64 = res, its residual r64 and the outer
    // squared-norm target stop64; the inner solve above works on (float) r64 with abs_stop
    const double *K64, *res;
    double *x64, *r64;
    double stop64;
};

// One linear solve's CG state, kept across launches when a solve pauses.
struct BState
{
    double rr, stop, alpha, beta, rr0, rr_final;
    int64_t it;       // iterations of the current (inner) CG solve
    int64_t it_total; // iterations of the whole linear solve (all refinements)
    int64_t status;   // bits: 1 iteration cap, 4 breakdown (p.Ap == 0), 8 paused at the end of the launch
    int32_t mode;     // 0 CG; refinement: 1 x64 += x32 next, 2 true residual next, 3 CG restarts next phase A
    int32_t refs;     // refinement steps finished (inner solves)
    int32_t caps;     // inner solves stopped by their cap
    int32_t pad;
    int64_t last_inner; // iterations of the last finished inner solve
};

struct BCtl
{
    unsigned bar; // barrier arrivals: starts at zero, only counts up
    int fail;     // a wait timed out
    int nact;     // problems in the launch
    int pad;
};

struct BArgs
{
    const BInst *inst;
    BState *st; // in: states of resumed solves; out (block 0, at the end): every problem's state
    BCtl *ctl;
    // [6][kMaxVirt] per-piece partials.  CG: 1 = p.Ap (phase A), 0 = ||r||^2 (phase B and the
    // start).  True residual of a refinement: 2, 3 in phase A and 4, 5 in phase B (||r64||^2,
    // ||(float) r64||^2).  Consecutive phases never write the same buffer, so a block one phase
    // ahead never overwrites partials another block still reads (the split, and with it the
    // slot of each piece, may change between two phases).
    double *part;
    int ninst;
    int64_t slice;   // iterations per launch; unfinished solves pause and resume later
};

// ---- block-wide integer scans / sums (deterministic)
template <typename T>
__device__ T block_exscan(T v, T *total, T *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
    for (int o = 1; o < 32; o <<= 1)
    {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        sh[w] = x;
    __syncthreads();
    if (w == 0)
    {
        T t = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : T(0);
        for (int o = 1; o < 32; o <<= 1)
        {
            const T y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o)
                t += y;
        }
        sh[lane] = t; // inclusive prefix of warp totals
    }
    __syncthreads();
    const T before = (w > 0 ? sh[w - 1] : T(0)) + x - v;
    *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

// The split.  The active problems' costs are laid end to end (rank order) and cut into
// gridDim.x equal segments, one per physical block: block b owns costs [b*C/G, (b+1)*C/G).
// A problem's piece in block b is its part of that segment, rounded to whole slices by the
// slices' starting cost (slice_off x (d^2 + 1)), so the pieces of one problem partition its
// slices; the update phases take the rows' unknowns in proportion, [s0*ndof/ns, s1*ndof/ns).
// Every SM carries the same matrix volume whatever the mix of sizes: a small problem shares a
// block with its neighbours in rank order, a large one spans many blocks.
__device__ __forceinline__ int seg_block(long long t, long long C, int G)
{
    // the last block b with b*C/G <= t
    const long long b = ((t + 1) * G + C - 1) / C - 1;
    return (int)(b < G - 1 ? b : G - 1);
}
__device__ __forceinline__ long long seg_bound(int b, long long C, int G) { return (long long)b * C / G; }

// first slice s with slice_off[s] >= v (slice_off strictly increasing, slice_off[ns] = slots)
__device__ __forceinline__ int slice_at(const int64_t *slice_off, int ns, long long v)
{
    int lo = 0, hi = ns;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (__ldg(slice_off + mid) >= v)
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo;
}

// What every block keeps of the launch: the CG scalars of each problem (indexed by problem), the
// rank tables of the active ones (rank r: problem act[r], cost prefix cum[r], pieces in blocks
// fb[r] .. fb[r] + g[r] - 1 whose partials sit at vs[r] ..) and this block's own pieces (ranks
// pr_lo .. pr_lo + np - 1, slices [ps0[k], ps1[k])).  All blocks apply the same decisions to
// the same totals, so the shared copies never differ.
struct BShared
{
    double rr[kMaxBatch], stop[kMaxBatch], alpha[kMaxBatch], beta[kMaxBatch], rrf[kMaxBatch];
    long long cit[kMaxBatch], itot[kMaxBatch], lastit[kMaxBatch];
    long long cum[kMaxBatch + 1];
    int status[kMaxBatch], mode[kMaxBatch], refs[kMaxBatch], caps[kMaxBatch];
    int act[kMaxBatch], g[kMaxBatch], vs[kMaxBatch], fb[kMaxBatch], keep[kMaxBatch];
    int ps0[kMaxBatch], ps1[kMaxBatch];
    int nact, nvirt, np, pr_lo;
    int scan[32];
    long long sum[32];
};

template <typename TV>
union BUnion
{
    TV red[32 * 3 * 32];         // phase A's column-split buffer
    double stage[3 * kMaxStage]; // the staged partials of a reduction (CG, ||r64||^2, ||(float) r64||^2)
    double wpart[kMaxBatch * 32]; // per (piece, warp) partials of a phase before the block's sums
};

constexpr size_t kBSharedBytes = ((sizeof(BShared) + 15) / 16) * 16;
template <typename TV>
constexpr size_t batch_smem_bytes()
{
    return kBSharedBytes + sizeof(BUnion<TV>);
}

// Recomputes the split over S.act[0 .. S.nact) and this block's pieces.  Whole block.
__device__ void batch_split(const BArgs &a, BShared &S)
{
    const int t = threadIdx.x, nact = S.nact, G = gridDim.x, b = blockIdx.x;
    const long long cost = (t < nact) ? a.inst[S.act[t]].cost : 0;
    long long C = 0;
    const long long before = block_exscan<long long>(cost, &C, S.sum);
    if (t < nact)
        S.cum[t] = before;
    if (t == 0)
        S.cum[nact] = C;
    __syncthreads();
    int g = 0, fb = 0;
    bool mine = false;
    if (t < nact)
    {
        fb = seg_block(S.cum[t], C, G);
        const int lb = seg_block(S.cum[t + 1] - 1, C, G);
        g = lb - fb + 1;
        mine = fb <= b && b <= lb;
    }
    int V = 0;
    const int vs = block_exscan<int>(g, &V, S.scan);
    if (t < nact)
    {
        S.g[t] = g;
        S.vs[t] = vs;
        S.fb[t] = fb;
    }
    if (t == 0)
    {
        S.nvirt = V;
        S.pr_lo = 0x7fffffff;
    }
    __syncthreads();
    if (mine)
        atomicMin(&S.pr_lo, t);
    const int np = __syncthreads_count(mine);
    if (t < np)
    {
        const int r = S.pr_lo + t;
        const BInst &I = a.inst[S.act[r]];
        const long long c0 = S.cum[r], c1 = S.cum[r + 1];
        const long long lo = max(seg_bound(b, C, G), c0) - c0;
        long long hi = min(seg_bound(b + 1, C, G), c1) - c0;
        if (hi < lo)
            hi = lo;
        const long long e1 = (long long)I.dim * I.dim + 1;
        S.ps0[t] = slice_at(I.slice_off, I.nslices, (lo + e1 - 1) / e1);
        S.ps1[t] = slice_at(I.slice_off, I.nslices, (hi + e1 - 1) / e1);
    }
    if (t == 0)
        S.np = np;
    __syncthreads();
}

// Counting grid barrier: barrier number `epoch` is passed once the word reaches
// (epoch + 1) * gridDim.x.  Bounded wait; false when it timed out (here or in another block).
__device__ bool batch_barrier(BCtl *ctl, unsigned &epoch, volatile int *s_fail)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        atomicAdd(&ctl->bar, 1u);
        const unsigned target = (epoch + 1u) * gridDim.x;
        const unsigned long long t0 = gtimer();
        while ((int)(ld_acquire(&ctl->bar) - target) < 0)
        {
            if (gtimer() - t0 > kBarrierTimeoutNs)
            {
                atomicExch(&ctl->fail, 1);
                *s_fail = 1;
                break;
            }
        }
        if (*reinterpret_cast<volatile int *>(&ctl->fail))
            *s_fail = 1;
    }
    epoch++;
    __syncthreads();
    return *s_fail == 0;
}

// fixed-order sum of rank r's partials (32-wide warp sums in piece order); whole warp
__device__ __forceinline__ double rank_total(const BShared &S, const double *stage, int r)
{
    const int lane = threadIdx.x & 31, g = S.g[r], vs = S.vs[r];
    double tot = 0;
    for (int c = 0; c < g; c += 32)
    {
        const double v = (c + lane < g) ? stage[vs + c + lane] : 0.0;
        tot += wsum(v);
    }
    return tot;
}

// A finished inner solve of a refining problem hands over to x64 += x32 (the next phase).
__device__ __forceinline__ void inner_done(BShared &S, int m, bool capped)
{
    S.lastit[m] = S.cit[m];
    S.refs[m] += 1;
    if (capped)
        S.caps[m] += 1;
    S.mode[m] = 1;
}

// After a barrier, in every block: reduce each active problem's partials, decide per problem,
// and re-split when problems left.  kind 0: after the start (||r||^2 of fresh solves); 1: after
// phase A (p.Ap -> alpha, or breakdown); 2: after phase B (||r||^2 -> beta, or converged /
// capped / paused).  Refining problems step through their own modes at every decision.
__device__ void batch_reduce_decide(const BArgs &a, BShared &S, int kind, int64_t it, double *stage)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double *part = a.part + (size_t)(kind == 1 ? 1 : 0) * kMaxVirt;
    const double *pr64 = a.part + (size_t)(kind == 1 ? 2 : 4) * kMaxVirt;
    const double *pb32 = pr64 + kMaxVirt;
    for (int v = threadIdx.x; v < S.nvirt; v += blockDim.x)
    {
        stage[v] = __ldcg(part + v);
        if (kind != 0)
        {
            stage[kMaxStage + v] = __ldcg(pr64 + v);
            stage[2 * kMaxStage + v] = __ldcg(pb32 + v);
        }
    }
    __syncthreads();
    for (int r = warp; r < S.nact; r += nw)
    {
        const int m = S.act[r];
        const bool resid = kind != 0 && S.mode[m] == 2;
        const double tot = rank_total(S, stage + (resid ? kMaxStage : 0), r);
        const double tot2 = resid ? rank_total(S, stage + 2 * kMaxStage, r) : 0.0;
        if (lane == 0)
        {
            const BInst &I = a.inst[m];
            int keep = 1;
            const int md = S.mode[m];
            if (kind == 0)
            {
                if (I.fresh)
                {
                    const double stop = (I.abs_stop >= 0) ? I.abs_stop : I.rtol * tot + I.atol;
                    S.rr[m] = tot;
                    S.stop[m] = stop;
                    S.beta[m] = 0.0;
                    S.cit[m] = 0;
                    S.rrf[m] = tot;
                    if (tot <= stop)
                    {
                        if (I.refine)
                            inner_done(S, m, false);
                        else
                            keep = 0;
                    }
                }
            }
            else if (md == 1)
                S.mode[m] = 2; // x64 += x32 ran in this phase; the true residual is next
            else if (md == 2)
            {
                // the true residual ran in this phase: tot = ||r64||^2, tot2 = ||(float) r64||^2
                S.rrf[m] = tot;
                if (tot <= I.stop64 || S.lastit[m] == 0 || S.refs[m] >= 30)
                    keep = 0;
                else
                {
                    S.rr[m] = tot2;
                    S.stop[m] = I.abs_stop;
                    S.beta[m] = 0.0;
                    S.cit[m] = 0;
                    S.mode[m] = (kind == 2) ? 0 : 3;
                }
            }
            else if (md == 3)
            {
                if (kind == 2)
                    S.mode[m] = 0;
            }
            else if (kind == 1)
            {
                if (tot == 0.0)
                {
                    S.status[m] |= 4;
                    S.rrf[m] = S.rr[m];
                    if (I.refine)
                        inner_done(S, m, false);
                    else
                        keep = 0;
                }
                else
                    S.alpha[m] = S.rr[m] / tot;
            }
            else
            {
                S.cit[m] += 1;
                S.itot[m] += 1;
                const bool done = tot <= S.stop[m];
                const bool capped = S.cit[m] >= I.maxit;
                S.rrf[m] = tot;
                if (done || capped)
                {
                    if (I.refine)
                        inner_done(S, m, !done);
                    else
                    {
                        if (!done)
                            S.status[m] |= 1;
                        keep = 0;
                    }
                }
                else
                {
                    S.beta[m] = tot / S.rr[m];
                    S.rr[m] = tot;
                }
            }
            // pause at the end of the launch's slice; only a solve in CG mode pauses (a refinement
            // step finishes first)
            if (keep && kind == 2 && S.mode[m] == 0 && it >= a.slice)
            {
                S.status[m] |= 8;
                keep = 0;
            }
            S.keep[r] = keep;
        }
    }
    __syncthreads();
    const int t = threadIdx.x, nact = S.nact;
    const int keep = (t < nact) ? S.keep[t] : 1;
    const int gone = __syncthreads_count(keep == 0);
    if (gone == 0)
        return;
    // compaction of the still-active ranks (order kept), then the new split
    const int mine = (t < nact) ? S.act[t] : -1;
    int nnew = 0;
    const int pos = block_exscan<int>((t < nact && keep) ? 1 : 0, &nnew, S.scan);
    if (t < nact && keep)
        S.keep[pos] = mine; // every thread has read its keep flag above
    __syncthreads();
    if (t < nnew)
        S.act[t] = S.keep[t];
    if (t == 0)
        S.nact = nnew;
    __syncthreads();
    batch_split(a, S);
}

// Only the FP32 variant runs inner solves of a refinement (FP64 items never refine).
template <typename TV>
constexpr bool kRefines = sizeof(TV) == 4;
// The FP64 variant deals each block's slices (phase A) and unknowns (phase B) of all its pieces
// to its warps as one list, with one block sync per phase (11% faster on the 64-plate batch).
// The FP32 variant keeps one block-wide pass and sum per piece: with the flat list its 80
// registers spill and it ran 27% slower.
template <typename TV>
constexpr bool kFlat = sizeof(TV) == 8;

// Refinement steps of a problem whose inner FP32 solve finished (the loop body of the mixed
// solve in cg.cu: x64 += x32, then r64 = res - K64 x64 and the next inner solve's start).
// x64 += x32 over the piece's unknowns
template <typename TV>
__device__ __forceinline__ void refine_add(const BInst &I, int s0, int s1)
{
    const int64_t lo = (int64_t)s0 * I.ndof / I.nslices, hi = (int64_t)s1 * I.ndof / I.nslices;
    const TV *x32 = static_cast<const TV *>(I.x);
    for (int64_t j = lo + threadIdx.x; j < hi; j += blockDim.x)
        I.x64[j] = I.x64[j] + (double)x32[j];
}

// For the rows of slices [s0, s1): r64 = res - K64 x64, then the inner solve's fresh start
// r32 = (float) r64, x32 = 0, p_old = 0.  Returns the thread's share of ||r64||^2 and, in *v2,
// of ||(float) r64||^2 (the inner solve's initial ||r||^2).
template <typename TV>
__device__ __forceinline__ double refine_residual(const BInst &I, int s0, int s1, uint64_t pf, uint64_t pl, double *v2)
{
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, D = I.dim;
    TV *x32 = static_cast<TV *>(I.x), *r32 = static_cast<TV *>(I.r), *pa = static_cast<TV *>(I.pa);
    double loc = 0, loc2 = 0;
    for (int sl = s0 + warp; sl < s1; sl += nw)
    {
        double acc[3];
        const int i = (D == 2) ? spmv_slice<double, double, 2>(sl, I.n, I.rowptr, I.perm, I.slice_off, I.col_sell,
                                                                I.K64, I.x64, I.x64, 0.0, acc, pf, pl)
                               : spmv_slice<double, double, 3>(sl, I.n, I.rowptr, I.perm, I.slice_off, I.col_sell,
                                                                I.K64, I.x64, I.x64, 0.0, acc, pf, pl);
        if (i >= 0)
            for (int c = 0; c < D; ++c)
            {
                const int64_t k = (int64_t)i * D + c;
                const double v = I.res[k] - acc[c];
                I.r64[k] = v;
                loc += v * v;
                const TV f = (TV)v;
                st_keep(r32 + k, f, pl);
                st_keep(x32 + k, TV(0), pl);
                st_keep(pa + k, TV(0), pl);
                loc2 += (double)f * (double)f;
            }
    }
    *v2 = loc2;
    return loc;
}

// One slice of phase A for a CG-mode problem: q = K p_new for its rows, p_new and q stored;
// returns the thread's share of p_new . q.  The same arithmetic as spmv_block's epilogue.
template <typename TK, typename TV, int D>
__device__ __forceinline__ double slice_cg(const BInst &I, int sl, TV beta, bool odd, uint64_t pf, uint64_t pl)
{
    const TV *pold = static_cast<const TV *>(odd ? I.pa : I.pb);
    TV *pnew = static_cast<TV *>(odd ? I.pb : I.pa);
    const TV *r = static_cast<const TV *>(I.r);
    TV *q = static_cast<TV *>(I.q);
    TV acc[D];
    const int i = spmv_slice<TK, TV, D, (sizeof(TV) == 4 ? 3 : 1)>(sl, I.n, I.rowptr, I.perm, I.slice_off, I.col_sell,
                                                                 static_cast<const TK *>(I.K), r, pold, beta, acc, pf,
                                                                 pl);
    double lpq = 0;
    if (i >= 0)
#pragma unroll
        for (int c = 0; c < D; ++c)
        {
            const int64_t k = (int64_t)i * D + c;
            const TV pn = ld_keep(r + k, pl) + beta * ld_keep(pold + k, pl);
            st_keep(pnew + k, pn, pl);
            st_keep(q + k, acc[c], pl);
            lpq += (double)pn * (double)acc[c];
        }
    return lpq;
}

// The partial of each CG-mode piece of this block: its warps' values (wpart[piece * 32 + warp])
// summed in warp order, one warp per piece, into dst at the piece's slot.
__device__ __forceinline__ void piece_sums(const BShared &S, const double *wpart, double *dst, int nw)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = warp; k < S.np; k += nw)
    {
        const int r = S.pr_lo + k;
        if (S.mode[S.act[r]] != 0)
            continue;
        const double tot = wsum(lane < nw ? wpart[k * 32 + lane] : 0.0);
        if (lane == 0)
            dst[S.vs[r] + (int)blockIdx.x - S.fb[r]] = tot;
    }
}

// Phase A of one piece: q = K p_new for its slices.  The FP32 variant (80 registers) keeps three
// steps of 2 x 2 blocks in flight per warp.
template <typename TK, typename TV, int D>
__device__ __forceinline__ double batch_spmv(const BInst *Ip, int s0, int s1, TV beta, bool odd, TV *red)
{
    const BInst &I = *Ip;
    const TV *pold = static_cast<const TV *>(odd ? I.pa : I.pb);
    TV *pnew = static_cast<TV *>(odd ? I.pb : I.pa);
    return spmv_block<TK, TV, D, (sizeof(TV) == 4 ? 3 : 1)>(s0, s1, I.n, I.rowptr, I.perm, I.slice_off, I.col_sell,
                                                             static_cast<const TK *>(I.K),
                                 static_cast<const TV *>(I.r), pold, pnew, static_cast<TV *>(I.q), beta,
                                 l2_evict_first(), l2_evict_last(), red);
}

// Threads per block: the FP32 variant runs 24 warps with up to 80 registers each, so its SpMV can
// keep several steps' loads in flight (2 x 2 FP32 blocks move only 16 bytes per lane and step);
// the FP64 variant keeps 32 warps at 64 registers, as the single-problem kernel does.
template <typename TV>
constexpr int kBatchThreads = sizeof(TV) == 4 ? 768 : kCGThreads;

template <typename TK, typename TV>
__global__ void __launch_bounds__(kBatchThreads<TV>, kCGMinBlocks) k_cg_batch(BArgs a)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    BShared &S = *reinterpret_cast<BShared *>(dsm);
    BUnion<TV> &U = *reinterpret_cast<BUnion<TV> *>(dsm + kBSharedBytes);
    __shared__ double sh[32];
    __shared__ int s_fail;
    TV *red = U.red;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31, nw = blockDim.x >> 5;
    if (t == 0)
    {
        s_fail = 0;
        S.nact = a.ninst;
    }
    for (int m = t; m < a.ninst; m += blockDim.x)
    {
        const BState &B = a.st[m];
        S.act[m] = m;
        S.rr[m] = B.rr;
        S.stop[m] = B.stop;
        S.alpha[m] = B.alpha;
        S.beta[m] = B.beta;
        S.rrf[m] = B.rr_final;
        S.cit[m] = B.it;
        S.itot[m] = B.it_total;
        S.lastit[m] = B.last_inner;
        S.status[m] = (int)B.status;
        S.mode[m] = B.mode;
        S.refs[m] = B.refs;
        S.caps[m] = B.caps;
    }
    __syncthreads();
    batch_split(a, S);
    unsigned epoch = 0;
    const uint64_t pf = l2_evict_first(), pl = l2_evict_last();
    double *const part0 = a.part, *const part1 = a.part + kMaxVirt;
    double *const partA = a.part + 2 * kMaxVirt, *const partB = a.part + 4 * kMaxVirt;

    // fresh solves: r = b, x = 0, p_old = 0; partial ||b||^2 (resumed solves keep their vectors)
    for (int k = 0; k < S.np; ++k)
    {
        const int r = S.pr_lo + k, m = S.act[r], pidx = S.vs[r] + (int)blockIdx.x - S.fb[r];
        const BInst &I = a.inst[m];
        double loc = 0;
        if (I.fresh)
        {
            const int64_t lo = (int64_t)S.ps0[k] * I.ndof / I.nslices, hi = (int64_t)S.ps1[k] * I.ndof / I.nslices;
            const TV *b = static_cast<const TV *>(I.b);
            TV *x = static_cast<TV *>(I.x), *rv = static_cast<TV *>(I.r), *pa = static_cast<TV *>(I.pa);
            for (int64_t j = lo + t; j < hi; j += blockDim.x)
            {
                const TV bv = b[j];
                st_keep(rv + j, bv, pl);
                st_keep(x + j, TV(0), pl);
                st_keep(pa + j, TV(0), pl);
                loc += (double)bv * (double)bv;
            }
        }
        block_partial_at(loc, part0 + pidx, sh);
    }
    if (!batch_barrier(a.ctl, epoch, &s_fail))
        return;
    batch_reduce_decide(a, S, 0, 0, U.stage);

    for (int64_t it = 1; S.nact > 0; ++it)
    {
        // phase A: q = K p_new (partials -> buffer 1); refining problems take their next step
        if constexpr (kRefines<TV>)
            for (int k = 0; k < S.np; ++k)
            {
                const int r = S.pr_lo + k, m = S.act[r], pidx = S.vs[r] + (int)blockIdx.x - S.fb[r];
                const int md = S.mode[m];
                if (md == 1)
                    refine_add<TV>(a.inst[m], S.ps0[k], S.ps1[k]);
                else if (md == 2)
                {
                    double v2 = 0;
                    const double v1 = refine_residual<TV>(a.inst[m], S.ps0[k], S.ps1[k], pf, pl, &v2);
                    block_partial_at(v1, partA + pidx, sh);
                    block_partial_at(v2, partA + kMaxVirt + pidx, sh);
                }
            }
        {
            int T = 0; // slices of this block's pieces in CG mode
            for (int k = 0; k < S.np; ++k)
                if (S.mode[S.act[S.pr_lo + k]] == 0)
                    T += S.ps1[k] - S.ps0[k];
            if (kFlat<TV> && 2 * T > nw)
            {
                // one list of all those slices, dealt round-robin to the warps across the pieces;
                // each warp leaves one partial per piece, summed per piece after one block sync
                int off = 0;
                for (int k = 0; k < S.np; ++k)
                {
                    const int m = S.act[S.pr_lo + k];
                    if (S.mode[m] != 0)
                        continue;
                    const BInst &I = a.inst[m];
                    const int nk = S.ps1[k] - S.ps0[k];
                    const bool odd = ((S.cit[m] + 1) & 1) != 0; // the solve's own iteration number
                    const TV beta = (TV)S.beta[m];
                    double lpq = 0;
                    for (int i = (warp - off % nw + nw) % nw; i < nk; i += nw)
                        lpq += (I.dim == 2) ? slice_cg<TK, TV, 2>(I, S.ps0[k] + i, beta, odd, pf, pl)
                                            : slice_cg<TK, TV, 3>(I, S.ps0[k] + i, beta, odd, pf, pl);
                    const double wv = wsum(lpq);
                    if (lane == 0)
                        U.wpart[k * 32 + warp] = wv;
                    off += nk;
                }
                __syncthreads();
                piece_sums(S, U.wpart, part1, nw);
            }
            else
                for (int k = 0; k < S.np; ++k)
                {
                    const int r = S.pr_lo + k, m = S.act[r], pidx = S.vs[r] + (int)blockIdx.x - S.fb[r];
                    if (S.mode[m] != 0)
                        continue;
                    const BInst &I = a.inst[m];
                    const bool odd = ((S.cit[m] + 1) & 1) != 0;
                    const double val = (I.dim == 2)
                                           ? batch_spmv<TK, TV, 2>(&I, S.ps0[k], S.ps1[k], (TV)S.beta[m], odd, red)
                                           : batch_spmv<TK, TV, 3>(&I, S.ps0[k], S.ps1[k], (TV)S.beta[m], odd, red);
                    block_partial_at(val, part1 + pidx, sh);
                }
        }
        if (!batch_barrier(a.ctl, epoch, &s_fail))
            return;
        batch_reduce_decide(a, S, 1, it, U.stage);
        // phase B: x += alpha p_new, r -= alpha q (partials -> buffer 0)
        for (int k = 0; k < S.np; ++k)
        {
            const int r = S.pr_lo + k, m = S.act[r], pidx = S.vs[r] + (int)blockIdx.x - S.fb[r];
            const BInst &I = a.inst[m];
            const int md = S.mode[m];
            if (md == 0)
            {
                const bool odd = ((S.cit[m] + 1) & 1) != 0;
                const TV al = (TV)S.alpha[m];
                const TV *pnew = static_cast<const TV *>(odd ? I.pb : I.pa);
                TV *x = static_cast<TV *>(I.x), *rv = static_cast<TV *>(I.r);
                const TV *q = static_cast<const TV *>(I.q);
                const int64_t lo = (int64_t)S.ps0[k] * I.ndof / I.nslices, hi = (int64_t)S.ps1[k] * I.ndof / I.nslices;
                double lrr = 0;
                for (int64_t j = lo + t; j < hi; j += blockDim.x)
                {
                    st_keep(x + j, ld_keep(x + j, pl) + al * ld_keep(pnew + j, pl), pl);
                    const TV rn = ld_keep(rv + j, pl) - al * ld_keep(q + j, pl);
                    st_keep(rv + j, rn, pl);
                    lrr += (double)rn * (double)rn;
                }
                if constexpr (kFlat<TV>)
                {
                    const double wv = wsum(lrr);
                    if (lane == 0)
                        U.wpart[k * 32 + warp] = wv;
                }
                else
                    block_partial_at(lrr, part0 + pidx, sh);
            }
            else if constexpr (kRefines<TV>)
            {
                if (md == 1)
                    refine_add<TV>(I, S.ps0[k], S.ps1[k]);
                else if (md == 2)
                {
                    double v2 = 0;
                    const double v1 = refine_residual<TV>(I, S.ps0[k], S.ps1[k], pf, pl, &v2);
                    block_partial_at(v1, partB + pidx, sh);
                    block_partial_at(v2, partB + kMaxVirt + pidx, sh);
                }
            }
        }
        if constexpr (kFlat<TV>)
        {
            __syncthreads();
            piece_sums(S, U.wpart, part0, nw);
        }
        if (!batch_barrier(a.ctl, epoch, &s_fail))
            return;
        batch_reduce_decide(a, S, 2, it, U.stage);
    }
    if (blockIdx.x == 0)
        for (int m = t; m < a.ninst; m += blockDim.x)
        {
            BState &B = a.st[m];
            B.rr = S.rr[m];
            B.stop = S.stop[m];
            B.alpha = S.alpha[m];
            B.beta = S.beta[m];
            B.rr_final = S.rrf[m];
            B.it = S.cit[m];
            B.it_total = S.itot[m];
            B.last_inner = S.lastit[m];
            B.status = S.status[m];
            B.mode = S.mode[m];
            B.refs = S.refs[m];
            B.caps = S.caps[m];
        }
}

// ---- single-reduction inner solves (the FP32 members of a refinement)
//
// The textbook CG needs two grid-wide reductions per iteration (p.Ap, then r.r), and in a batch
// whose members are small each reduction costs a grid barrier plus every block's decision pass:
// the floor of a batched iteration.  The FP32 inner solves of mixed members therefore run the
// Chronopoulos-Gear form of the same CG (the same iterates in exact arithmetic, one reduction
// per iteration), with w = A r computed and s = A p kept by recurrence:
//   p_k = r_k + beta_{k-1} p_{k-1},   s_k = w_k + beta_{k-1} s_{k-1},
//   x_{k+1} = x_k + alpha_k p_k,      r_{k+1} = r_k - alpha_k s_k,      w_{k+1} = A r_{k+1},
//   gamma_{k+1} = r_{k+1}.r_{k+1} and delta_{k+1} = w_{k+1}.r_{k+1} in one reduction,
//   beta_k = gamma_{k+1} / gamma_k,   alpha_{k+1} = gamma_{k+1} / (delta_{k+1} - beta_k gamma_{k+1} / alpha_k).
// The SpMV gathers the neighbours' r_{k+1} formed on the fly from their r_k, w_k and s_{k-1},
// so r, w and s alternate between two buffers each (the iteration's parity).  Every inner solve
// opens with one phase w_0 = A r_0, alpha_0 = gamma_0 / delta_0.  The FP64 refinement around it
// (x64 += x32, the true residual, the restart) and its stopping rule are those of k_cg_batch.
//
// Modes of a member (S.mode): 6 open a fresh solve from b; 3 open an inner solve from r (after a
// true residual); 0 iterate; 1 x64 += x32 next; 2 the true residual next.

// q = K v for the row at this lane of slice sl, with v gathered as r (INIT) or formed on the fly
// as r - alpha (w + beta s) from the three buffers; returns the particle id (-1 past the end).
template <int D, int U, bool INIT>
__device__ __forceinline__ int sr_spmv_slice(int sl, const BInst &I, const float *__restrict__ r,
                                             const float *__restrict__ w, const float *__restrict__ sv, float alpha,
                                             float beta, float acc[D], uint64_t pf, uint64_t pl, int k0, int kstep)
{
    constexpr int E = D * D;
    const int lane = threadIdx.x & 31;
    const int pos = sl * kSlice + lane;
    const bool valid = pos < I.n;
    const int i = valid ? I.perm[pos] : -1;
    const int myn = valid ? (I.rowptr[i + 1] - I.rowptr[i]) : 0;
    const int64_t off = I.slice_off[sl];
    const int wd = (int)(I.slice_off[sl + 1] - off);
    const int *cp = I.col_sell + off * kSlice + lane;
    const float *kp = static_cast<const float *>(I.K) + off * E * kSlice + lane;
#pragma unroll
    for (int k = 0; k < D; ++k)
        acc[k] = 0.0f;
    int jn[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
    {
        const int kk = k0 + u * kstep;
        jn[u] = (kk < myn) ? ld_stream(cp + (int64_t)kk * kSlice, pf) : 0;
    }
    for (int k = k0; k < wd; k += U * kstep)
    {
        int j[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            j[u] = jn[u];
            const int kk = k + (U + u) * kstep;
            jn[u] = (kk < myn) ? ld_stream(cp + (int64_t)kk * kSlice, pf) : 0;
        }
        float xv[U][D], kv[U][E];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int kk = k + u * kstep;
            if (kk < myn)
            {
                if constexpr (D == 2)
                {
                    const int64_t q = (int64_t)j[u] * 2;
                    const float2 rv = ld_keep2(r + q, pl);
                    if (INIT)
                    {
                        xv[u][0] = rv.x;
                        xv[u][1] = rv.y;
                    }
                    else
                    {
                        const float2 wv = ld_keep2(w + q, pl), s2 = ld_keep2(sv + q, pl);
                        xv[u][0] = rv.x - alpha * (wv.x + beta * s2.x);
                        xv[u][1] = rv.y - alpha * (wv.y + beta * s2.y);
                    }
                }
                else
#pragma unroll
                    for (int c = 0; c < D; ++c)
                    {
                        const int64_t q = (int64_t)j[u] * D + c;
                        if (INIT)
                            xv[u][c] = ld_keep(r + q, pl);
                        else
                            xv[u][c] = ld_keep(r + q, pl) - alpha * (ld_keep(w + q, pl) + beta * ld_keep(sv + q, pl));
                    }
                const float *kb = kp + (int64_t)kk * E * kSlice;
#pragma unroll
                for (int e = 0; e < E; ++e)
                    kv[u][e] = ld_stream(kb + e * kSlice, pf);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k + u * kstep < myn)
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c)
                        acc[rr] += kv[u][rr * D + c] * xv[u][c];
    }
    return i;
}

// The vector work of one row after its SpMV (acc = K v): the opening (INIT: r_0, w_0 = A r_0 and
// the zeroed x, p, s_{-1}; gamma_0, delta_0) or iteration k of parity cur (s_k, p_k, x_{k+1},
// r_{k+1}, w_{k+1}; gamma_{k+1}, delta_{k+1}), accumulated into lg, ld.
template <int D, bool INIT>
__device__ __forceinline__ void sr_row(const BInst &I, int i, const float *acc, int cur, bool fresh, float alpha,
                                       float beta, uint64_t pl, double &lg, double &ld)
{
    if (i < 0)
        return;
    float *x = static_cast<float *>(I.x), *p = static_cast<float *>(I.pa);
    float *r0 = static_cast<float *>(I.r), *r1 = static_cast<float *>(I.r1);
    float *w0 = static_cast<float *>(I.q), *w1 = static_cast<float *>(I.w1);
    float *s0b = static_cast<float *>(I.pb), *s1b = static_cast<float *>(I.s1);
    // this iteration's buffers by parity: r_k, w_k in rc, wc; s_{k-1} in sp; s_k goes to sc,
    // r_{k+1} to rn_, w_{k+1} to wn
    float *rc = cur ? r1 : r0, *rn_ = cur ? r0 : r1, *wc = cur ? w1 : w0, *wn = cur ? w0 : w1;
    float *sc = cur ? s1b : s0b, *sp = cur ? s0b : s1b;
    if constexpr (D == 2)
        if (!INIT)
        {
            // the same arithmetic on both components, each vector moved 8 bytes at a time
            const int64_t k = (int64_t)i * 2;
            const float2 w2 = ld_keep2(wc + k, pl), s2 = ld_keep2(sp + k, pl), r2 = ld_keep2(rc + k, pl);
            const float2 p2 = ld_keep2(p + k, pl), x2 = ld_keep2(x + k, pl);
            const float2 sk = make_float2(w2.x + beta * s2.x, w2.y + beta * s2.y);
            const float2 pk = make_float2(r2.x + beta * p2.x, r2.y + beta * p2.y);
            st_keep2(x + k, make_float2(x2.x + alpha * pk.x, x2.y + alpha * pk.y), pl);
            const float2 rn = make_float2(r2.x - alpha * sk.x, r2.y - alpha * sk.y);
            st_keep2(sc + k, sk, pl);
            st_keep2(p + k, pk, pl);
            st_keep2(rn_ + k, rn, pl);
            st_keep2(wn + k, make_float2(acc[0], acc[1]), pl);
            lg += (double)rn.x * (double)rn.x;
            ld += (double)acc[0] * (double)rn.x;
            lg += (double)rn.y * (double)rn.y;
            ld += (double)acc[1] * (double)rn.y;
            return;
        }
#pragma unroll
    for (int c = 0; c < D; ++c)
    {
        const int64_t k = (int64_t)i * D + c;
        if (INIT)
        {
            const float v = ld_keep((fresh ? static_cast<const float *>(I.b) : r0) + k, pl);
            if (fresh)
                st_keep(r0 + k, v, pl);
            st_keep(w0 + k, acc[c], pl);
            st_keep(x + k, 0.0f, pl);
            st_keep(p + k, 0.0f, pl);
            st_keep(s1b + k, 0.0f, pl);
            lg += (double)v * (double)v;
            ld += (double)acc[c] * (double)v;
        }
        else
        {
            const float sk = ld_keep(wc + k, pl) + beta * ld_keep(sp + k, pl);
            const float rk = ld_keep(rc + k, pl);
            const float pk = rk + beta * ld_keep(p + k, pl);
            st_keep(x + k, ld_keep(x + k, pl) + alpha * pk, pl);
            const float rn = rk - alpha * sk;
            st_keep(sc + k, sk, pl);
            st_keep(p + k, pk, pl);
            st_keep(rn_ + k, rn, pl);
            st_keep(wn + k, acc[c], pl);
            lg += (double)rn * (double)rn;
            ld += (double)acc[c] * (double)rn;
        }
    }
}

// the gathered sources of a phase: the opening reads b (fresh) or r_0; an iteration reads r_k,
// w_k and s_{k-1}
__device__ __forceinline__ void sr_sources(const BInst &I, bool init, int cur, bool fresh, const float **gr,
                                           const float **gw, const float **gs)
{
    const float *r0 = static_cast<const float *>(I.r), *r1 = static_cast<const float *>(I.r1);
    const float *w0 = static_cast<const float *>(I.q), *w1 = static_cast<const float *>(I.w1);
    const float *s0b = static_cast<const float *>(I.pb), *s1b = static_cast<const float *>(I.s1);
    *gr = init ? (fresh ? static_cast<const float *>(I.b) : r0) : (cur ? r1 : r0);
    *gw = cur ? w1 : w0;
    *gs = cur ? s0b : s1b;
}

// One slice of a piece by one warp (the flat work list of k_cg_batch_sr).
template <int D, bool INIT, int UV>
__device__ __forceinline__ void sr_slice(const BInst &I, int sl, int cur, bool fresh, float alpha, float beta,
                                         uint64_t pf, uint64_t pl, double &lg, double &ld)
{
    constexpr int U = (D == 2) ? UV : 1;
    const float *gr, *gw, *gs;
    sr_sources(I, INIT, cur, fresh, &gr, &gw, &gs);
    float acc[D];
    const int i = sr_spmv_slice<D, U, INIT>(sl, I, gr, gw, gs, alpha, beta, acc, pf, pl, 0, 1);
    sr_row<D, INIT>(I, i, acc, cur, fresh, alpha, beta, pl, lg, ld);
}

// ---- the bulk-copy-fed SpMV of the single-reduction kernel (kernel 3)
//
// In a flat phase each warp walks its slices of a piece; the register-fed SpMV waits on the
// matrix loads of every step (one DRAM latency per 2 x 2 step pair), which held the 64-plate
// batch at about a quarter of HBM bandwidth.  Here the warp's lane 0 streams its slices' block
// values and columns into two shared-memory chunk buffers with bulk asynchronous copies, two
// chunks ahead, each completed on its own mbarrier; the lanes read values and columns from shared
// memory and only the vector gathers (mostly L1/L2 hits) remain on the critical path.  A chunk is
// kPipeSlots<D> block slots of one slice: D = 2: 8 x (4 values + 1 column) x 128 bytes; D = 3:
// 4 x (9 + 1) x 128 bytes; both about 5 KB per buffer.  Per warp the region holds the two value
// buffers, the two column buffers and the two mbarriers.
template <int D>
constexpr int kPipeSlots = D == 2 ? 8 : 4;
// the FP64 true residual of a refinement streams K64: half the slots per chunk in the same bytes
template <int D>
constexpr int kPipeSlots64 = kPipeSlots<D> / 2;
template <int D>
constexpr int kPipeValBytes = kPipeSlots<D> * D * D * kSlice * 4; // one value buffer
constexpr int kPipeBarOff = 10240;   // the two mbarriers, after the buffers of either dimension
constexpr int kPipeWarpBytes = 10368; // per warp, a multiple of 128
static_assert(2 * kPipeValBytes<2> + 2 * kPipeSlots<2> * kSlice * 4 == kPipeBarOff, "2D buffers");
static_assert(2 * kPipeValBytes<3> + 2 * kPipeSlots<3> * kSlice * 4 == kPipeBarOff, "3D buffers");
constexpr int kSrPipeThreads = 384;

struct SrPipe
{
    unsigned char *base; // this warp's region
    uint32_t n;          // chunks issued so far by this warp: chunk m uses buffer m & 1, phase m >> 1
    bool ok;             // false after a wait ran out of time
};

template <typename V, int D>
__device__ __forceinline__ V *pipe_vals(const SrPipe &P, uint32_t m)
{
    return reinterpret_cast<V *>(P.base + (m & 1) * kPipeValBytes<D>);
}
template <int D>
__device__ __forceinline__ int *pipe_cols(const SrPipe &P, uint32_t m)
{
    return reinterpret_cast<int *>(P.base + 2 * kPipeValBytes<D>) + (m & 1) * kPipeSlots<D> * kSlice;
}
__device__ __forceinline__ uint64_t *pipe_bar(const SrPipe &P, uint32_t m)
{
    return reinterpret_cast<uint64_t *>(P.base + kPipeBarOff) + (m & 1);
}

// Waits for chunk m's copies (whole warp).  When the wait runs out of time: a bounded wait for the
// warp's later copies still in flight, P.ok = false, and false.
__device__ __forceinline__ bool pipe_wait(SrPipe &P, uint32_t m)
{
    const bool ok = mbar_wait_bounded(pipe_bar(P, m), (m >> 1) & 1, kBarrierTimeoutNs);
    if (__all_sync(0xffffffffu, ok))
        return true;
    for (uint32_t q = m + 1; q < P.n; ++q)
        mbar_wait_bounded(pipe_bar(P, q), (q >> 1) & 1, kBarrierTimeoutNs / 4);
    P.ok = false;
    return false;
}

// The issue cursor over a warp's chunks: slices s, s + step, ... < end, chunks of each slice.
struct SrCursor
{
    int sl, step, end, c0, wd;
    int64_t off;
};

__device__ __forceinline__ void cursor_load(const BInst &I, SrCursor &c)
{
    while (c.sl < c.end)
    {
        c.off = I.slice_off[c.sl];
        c.wd = (int)(I.slice_off[c.sl + 1] - c.off);
        if (c.wd > 0)
            return;
        c.sl += c.step;
    }
}

// Issues the cursor's next chunk (lane 0), if any, and advances the cursor: C block slots of
// values (V) from Kg and their columns.  Whole warp.
template <typename V, int D, int C>
__device__ __forceinline__ void pipe_issue_next(const BInst &I, const V *Kg, SrPipe &P, SrCursor &c, uint64_t pf)
{
    constexpr int E = D * D;
    if (c.sl >= c.end)
        return;
    const int cn = min(C, c.wd - c.c0);
    if ((threadIdx.x & 31) == 0)
    {
        // the lanes' reads of the buffer (ordered before this lane by the caller's __syncwarp)
        // come before the copy's writes into it
        fence_proxy_async_smem();
        uint64_t *bar = pipe_bar(P, P.n);
        const uint32_t vb = (uint32_t)(cn * E * kSlice * sizeof(V)), cb = (uint32_t)cn * kSlice * 4;
        mbar_arrive_expect_tx(bar, vb + cb);
        bulk_g2s(pipe_vals<V, D>(P, P.n), Kg + (c.off + c.c0) * E * kSlice, vb, bar, pf);
        bulk_g2s(pipe_cols<D>(P, P.n), I.col_sell + (c.off + c.c0) * kSlice, cb, bar, pf);
    }
    P.n++;
    c.c0 += C;
    if (c.c0 >= c.wd)
    {
        c.c0 = 0;
        c.sl += c.step;
        cursor_load(I, c);
    }
}

// A slice's offsets and the lane's row, loaded one slice ahead of its use: meta_begin issues the
// offsets and the row id, meta_finish (after the current slice's chunks) the row's length.
struct SliceMeta
{
    int64_t off;
    int wd, i, myn;
};

__device__ __forceinline__ void meta_begin(const BInst &I, int sl, int end, SliceMeta &m)
{
    if (sl >= end)
        return;
    m.off = I.slice_off[sl];
    m.wd = (int)(I.slice_off[sl + 1] - m.off);
    const int pos = sl * kSlice + (threadIdx.x & 31);
    m.i = pos < I.n ? I.perm[pos] : -1;
}

__device__ __forceinline__ void meta_finish(const BInst &I, SliceMeta &m)
{
    m.myn = m.i >= 0 ? (I.rowptr[m.i + 1] - I.rowptr[m.i]) : 0;
}

// The warp's slices s_first, s_first + s_step, ... < s_end of one piece in one phase (the work
// of sr_slice for each), their block values and columns arriving by bulk copies.
template <int D, bool INIT>
__device__ void sr_slices_pipe(const BInst &I, int s_first, int s_step, int s_end, int cur, bool fresh, float alpha,
                               float beta, uint64_t pf, uint64_t pl, double &lg, double &ld, SrPipe &P)
{
    constexpr int E = D * D, C = kPipeSlots<D>;
    if (s_first >= s_end || !P.ok)
        return;
    const int lane = threadIdx.x & 31;
    const float *gr, *gw, *gs;
    sr_sources(I, INIT, cur, fresh, &gr, &gw, &gs);
    SrCursor cur_i{s_first, s_step, s_end, 0, 0, 0};
    cursor_load(I, cur_i);
    uint32_t m = P.n; // next chunk to consume
    const float *Kg = static_cast<const float *>(I.K);
    pipe_issue_next<float, D, C>(I, Kg, P, cur_i, pf);
    pipe_issue_next<float, D, C>(I, Kg, P, cur_i, pf);
    SliceMeta cm{0, 0, -1, 0}, nm{0, 0, -1, 0};
    meta_begin(I, s_first, s_end, cm);
    meta_finish(I, cm);
    for (int sl = s_first; sl < s_end; sl += s_step)
    {
        const int wd = cm.wd, i = cm.i, myn = cm.myn;
        meta_begin(I, sl + s_step, s_end, nm);
        float acc[D];
#pragma unroll
        for (int c = 0; c < D; ++c)
            acc[c] = 0.0f;
        for (int c0 = 0; c0 < wd; c0 += C)
        {
            const int cn = min(C, wd - c0);
            if (!pipe_wait(P, m))
                return;
            const float *kv = pipe_vals<float, D>(P, m);
            const int *cv = pipe_cols<D>(P, m);
            float xv[C][D];
#pragma unroll
            for (int t = 0; t < C; ++t)
                if (t < cn && c0 + t < myn)
                {
                    const int j = cv[t * kSlice + lane];
                    if constexpr (D == 2)
                    {
                        // a 2D particle's two components in one 8-byte load per vector
                        const int64_t q = (int64_t)j * 2;
                        const float2 rv = ld_keep2(gr + q, pl);
                        if (INIT)
                        {
                            xv[t][0] = rv.x;
                            xv[t][1] = rv.y;
                        }
                        else
                        {
                            const float2 wv = ld_keep2(gw + q, pl), sv = ld_keep2(gs + q, pl);
                            xv[t][0] = rv.x - alpha * (wv.x + beta * sv.x);
                            xv[t][1] = rv.y - alpha * (wv.y + beta * sv.y);
                        }
                    }
                    else
#pragma unroll
                        for (int c = 0; c < D; ++c)
                        {
                            const int64_t q = (int64_t)j * D + c;
                            if (INIT)
                                xv[t][c] = ld_keep(gr + q, pl);
                            else
                                xv[t][c] =
                                    ld_keep(gr + q, pl) - alpha * (ld_keep(gw + q, pl) + beta * ld_keep(gs + q, pl));
                        }
                }
#pragma unroll
            for (int t = 0; t < C; ++t)
                if (t < cn && c0 + t < myn)
#pragma unroll
                    for (int rr = 0; rr < D; ++rr)
#pragma unroll
                        for (int c = 0; c < D; ++c)
                            acc[rr] += kv[(t * E + rr * D + c) * kSlice + lane] * xv[t][c];
            ++m;
            __syncwarp();
            // the buffer just read takes the chunk two ahead
            pipe_issue_next<float, D, C>(I, Kg, P, cur_i, pf);
        }
        if (sl + s_step < s_end)
            meta_finish(I, nm);
        sr_row<D, INIT>(I, i, acc, cur, fresh, alpha, beta, pl, lg, ld);
        cm = nm;
    }
}

// The true residual of a refinement for the warp's slices s_first, s_first + s_step, ... < s_end
// of one piece (the work of refine_residual for each row: r64 = res - K64 x64, then r32 =
// (float) r64, x32 = 0, p = 0), the FP64 block values and columns arriving by bulk copies.  The
// thread's shares of ||r64||^2 and ||(float) r64||^2 are added to v1, v2.
template <int D>
__device__ void res_slices_pipe(const BInst &I, int s_first, int s_step, int s_end, uint64_t pf, uint64_t pl, double &v1,
                                double &v2, SrPipe &P)
{
    constexpr int E = D * D, C = kPipeSlots64<D>;
    if (s_first >= s_end || !P.ok)
        return;
    const int lane = threadIdx.x & 31;
    float *x32 = static_cast<float *>(I.x), *r32 = static_cast<float *>(I.r), *pa = static_cast<float *>(I.pa);
    SrCursor cur_i{s_first, s_step, s_end, 0, 0, 0};
    cursor_load(I, cur_i);
    uint32_t m = P.n;
    const double *Kg = I.K64;
    pipe_issue_next<double, D, C>(I, Kg, P, cur_i, pf);
    pipe_issue_next<double, D, C>(I, Kg, P, cur_i, pf);
    SliceMeta cm{0, 0, -1, 0}, nm{0, 0, -1, 0};
    meta_begin(I, s_first, s_end, cm);
    meta_finish(I, cm);
    for (int sl = s_first; sl < s_end; sl += s_step)
    {
        const int wd = cm.wd, i = cm.i, myn = cm.myn;
        meta_begin(I, sl + s_step, s_end, nm);
        double acc[D];
#pragma unroll
        for (int c = 0; c < D; ++c)
            acc[c] = 0.0;
        for (int c0 = 0; c0 < wd; c0 += C)
        {
            const int cn = min(C, wd - c0);
            if (!pipe_wait(P, m))
                return;
            const double *kv = pipe_vals<double, D>(P, m);
            const int *cv = pipe_cols<D>(P, m);
            double xv[C][D];
#pragma unroll
            for (int t = 0; t < C; ++t)
                if (t < cn && c0 + t < myn)
                {
                    const int j = cv[t * kSlice + lane];
                    if constexpr (D == 2)
                    {
                        const double2 v = ld_keep2(I.x64 + (int64_t)j * 2, pl);
                        xv[t][0] = v.x;
                        xv[t][1] = v.y;
                    }
                    else
#pragma unroll
                        for (int c = 0; c < D; ++c)
                            xv[t][c] = ld_keep(I.x64 + (int64_t)j * D + c, pl);
                }
#pragma unroll
            for (int t = 0; t < C; ++t)
                if (t < cn && c0 + t < myn)
#pragma unroll
                    for (int rr = 0; rr < D; ++rr)
#pragma unroll
                        for (int c = 0; c < D; ++c)
                            acc[rr] += kv[(t * E + rr * D + c) * kSlice + lane] * xv[t][c];
            ++m;
            __syncwarp();
            pipe_issue_next<double, D, C>(I, Kg, P, cur_i, pf);
        }
        if (sl + s_step < s_end)
            meta_finish(I, nm);
        if (i >= 0)
#pragma unroll
            for (int c = 0; c < D; ++c)
            {
                const int64_t k = (int64_t)i * D + c;
                const double v = I.res[k] - acc[c];
                I.r64[k] = v;
                v1 += v * v;
                const float f = (float)v;
                st_keep(r32 + k, f, pl);
                st_keep(x32 + k, 0.0f, pl);
                st_keep(pa + k, 0.0f, pl);
                v2 += (double)f * (double)f;
            }
        cm = nm;
    }
}

// One phase of a member's piece (slices [s0, s1)) in mode 0 (INIT false: iteration k of parity
// cur) or mode 3/6 (INIT: w_0 = A r_0, the solve's opening; fresh: r_0 = b).  Whole block; with
// fewer slices than warps several warps share a slice (column split through `red`).  Returns
// the thread's shares of gamma (r.r) and, in *ldelta, of delta (w.r).
template <int D, bool INIT, int UV>
__device__ __forceinline__ double sr_phase(const BInst &I, int s0, int s1, int cur, bool fresh, float alpha, float beta,
                                           uint64_t pf, uint64_t pl, float *red, double *ldelta)
{
    constexpr int U = (D == 2) ? UV : 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const float *gr, *gw, *gs;
    sr_sources(I, INIT, cur, fresh, &gr, &gw, &gs);
    double lg = 0, ld = 0;
    const int ns = s1 - s0;
    if (ns > 0)
    {
        if (2 * ns > nw)
        {
            for (int sl = s0 + warp; sl < s1; sl += nw)
            {
                float acc[D];
                const int i = sr_spmv_slice<D, U, INIT>(sl, I, gr, gw, gs, alpha, beta, acc, pf, pl, 0, 1);
                sr_row<D, INIT>(I, i, acc, cur, fresh, alpha, beta, pl, lg, ld);
            }
        }
        else
        {
            int S = 2;
            while (S < kMaxColumnSplit && ns * S * 2 <= nw)
                S *= 2;
            const int ls = warp / S, part = warp % S;
            float acc[D];
#pragma unroll
            for (int c = 0; c < D; ++c)
                acc[c] = 0.0f;
            int i = -1;
            if (ls < ns)
                i = sr_spmv_slice<D, U, INIT>(s0 + ls, I, gr, gw, gs, alpha, beta, acc, pf, pl, part, S);
            if (ls < ns && part > 0)
#pragma unroll
                for (int c = 0; c < D; ++c)
                    red[(warp * D + c) * 32 + lane] = acc[c];
            __syncthreads();
            if (ls < ns && part == 0)
            {
                for (int q = 1; q < S; ++q)
#pragma unroll
                    for (int c = 0; c < D; ++c)
                        acc[c] += red[((warp + q) * D + c) * 32 + lane];
                sr_row<D, INIT>(I, i, acc, cur, fresh, alpha, beta, pl, lg, ld);
            }
            __syncthreads();
        }
    }
    *ldelta = ld;
    return lg;
}

// After the barrier of phase `ph`, in every block: each active member's gamma and delta (or its
// true residual's two norms), its decision, and the compaction / re-split when members left.
__device__ void sr_reduce_decide(const BArgs &a, BShared &S, int64_t ph, double *stage)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double *p0 = a.part + (size_t)(2 * (ph & 1)) * kMaxVirt, *p1 = p0 + kMaxVirt;
    for (int v = threadIdx.x; v < S.nvirt; v += blockDim.x)
    {
        stage[v] = __ldcg(p0 + v);
        stage[kMaxStage + v] = __ldcg(p1 + v);
    }
    __syncthreads();
    for (int r = warp; r < S.nact; r += nw)
    {
        const int m = S.act[r];
        const int md = S.mode[m];
        const bool sums = md != 1;
        const double g = sums ? rank_total(S, stage, r) : 0.0;
        const double d = sums ? rank_total(S, stage + kMaxStage, r) : 0.0;
        if (lane == 0)
        {
            const BInst &I = a.inst[m];
            int keep = 1;
            if (md == 6 || md == 3)
            {
                // the opening phase: gamma_0 = r_0.r_0, delta_0 = (A r_0).r_0
                if (md == 6)
                {
                    S.stop[m] = (I.abs_stop >= 0) ? I.abs_stop : I.rtol * g + I.atol;
                    S.cit[m] = 0;
                }
                S.rr[m] = g;
                S.rrf[m] = g;
                S.beta[m] = 0.0;
                if (g <= S.stop[m])
                {
                    if (I.refine)
                        inner_done(S, m, false);
                    else
                        keep = 0;
                }
                else if (d == 0.0)
                {
                    S.status[m] |= 4;
                    if (I.refine)
                        inner_done(S, m, false);
                    else
                        keep = 0;
                }
                else
                {
                    S.alpha[m] = g / d;
                    S.mode[m] = 0;
                }
            }
            else if (md == 1)
                S.mode[m] = 2; // x64 += x32 ran; the true residual is next
            else if (md == 2)
            {
                // the true residual ran: g = ||r64||^2, d = ||(float) r64||^2 (the next r_0)
                S.rrf[m] = g;
                if (g <= I.stop64 || S.lastit[m] == 0 || S.refs[m] >= 30)
                    keep = 0;
                else
                {
                    S.stop[m] = I.abs_stop;
                    S.cit[m] = 0;
                    S.mode[m] = 3;
                }
            }
            else
            {
                // iteration k ran: g = gamma_{k+1}, d = delta_{k+1}
                S.cit[m] += 1;
                S.itot[m] += 1;
                S.rrf[m] = g;
                const bool done = g <= S.stop[m];
                const bool capped = S.cit[m] >= I.maxit;
                if (done || capped)
                {
                    if (I.refine)
                        inner_done(S, m, !done);
                    else
                    {
                        if (!done)
                            S.status[m] |= 1;
                        keep = 0;
                    }
                }
                else
                {
                    const double beta = g / S.rr[m];
                    const double den = d - beta * g / S.alpha[m];
                    if (den == 0.0)
                    {
                        S.status[m] |= 4;
                        if (I.refine)
                            inner_done(S, m, false);
                        else
                            keep = 0;
                    }
                    else
                    {
                        S.beta[m] = beta;
                        S.alpha[m] = g / den;
                        S.rr[m] = g;
                    }
                }
            }
            // pause at the end of the launch's slice; only an iterating solve pauses
            if (keep && S.mode[m] == 0 && ph + 1 >= a.slice)
            {
                S.status[m] |= 8;
                keep = 0;
            }
            S.keep[r] = keep;
        }
    }
    __syncthreads();
    const int t = threadIdx.x, nact = S.nact;
    const int keep = (t < nact) ? S.keep[t] : 1;
    const int gone = __syncthreads_count(keep == 0);
    if (gone == 0)
        return;
    const int mine = (t < nact) ? S.act[t] : -1;
    int nnew = 0;
    const int pos = block_exscan<int>((t < nact && keep) ? 1 : 0, &nnew, S.scan);
    if (t < nact && keep)
        S.keep[pos] = mine;
    __syncthreads();
    if (t < nnew)
        S.act[t] = S.keep[t];
    if (t == 0)
        S.nact = nnew;
    __syncthreads();
    batch_split(a, S);
}

// UV: 2 x 2 FP32 steps in flight per warp in the 2D SpMV (1 or 2); 2 needs 128 registers, so its
// blocks have 512 threads, against 768 at 80 registers for 1.  PIPE: the flat phases' SpMV is fed by
// bulk copies (sr_slices_pipe; 384 threads at up to 168 registers, the 8-slot chunks' gathers in
// flight without spills; each warp with its region after the shared state).
template <int UV>
constexpr int kSrThreads = UV == 2 ? 512 : 768;
// Kernel 3 keeps only the first kPipeFlatPieces x 64 doubles of the union's per-(piece, warp)
// partials (a flat phase needs np <= kPipeFlatPieces), so its union ends with the staged partials
// and the warps' copy buffers follow.
constexpr int kPipeFlatPieces = 16;
constexpr size_t kPipeUnionBytes = sizeof(double) * 3 * kMaxStage;
static_assert(kPipeUnionBytes >= sizeof(float) * 32 * 3 * 32 && kPipeUnionBytes >= sizeof(double) * kPipeFlatPieces * 64,
              "the union's other members fit");
constexpr size_t kSrPipeOffset = ((sizeof(BShared) + 15) / 16 * 16 + kPipeUnionBytes + 127) / 128 * 128;
static_assert(kSrPipeOffset + (kSrPipeThreads / 32) * kPipeWarpBytes <= 232448, "shared memory of kernel 3");

template <int UV, bool PIPE>
__global__ void __launch_bounds__(PIPE ? kSrPipeThreads : kSrThreads<UV>, kCGMinBlocks) k_cg_batch_sr(BArgs a)
{
    extern __shared__ __align__(128) unsigned char dsm[];
    BShared &S = *reinterpret_cast<BShared *>(dsm);
    BUnion<float> &Un = *reinterpret_cast<BUnion<float> *>(dsm + kBSharedBytes);
    __shared__ double sh[32];
    __shared__ int s_fail;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31, nw = blockDim.x >> 5;
    SrPipe pipe{dsm + kSrPipeOffset + (size_t)warp * kPipeWarpBytes, 0u, true};
    if constexpr (PIPE)
        if (lane == 0)
        {
            mbar_init(pipe_bar(pipe, 0), 1);
            mbar_init(pipe_bar(pipe, 1), 1);
            mbar_init_fence();
        }
    if (t == 0)
    {
        s_fail = 0;
        S.nact = a.ninst;
    }
    for (int m = t; m < a.ninst; m += blockDim.x)
    {
        const BState &B = a.st[m];
        const BInst &I = a.inst[m];
        S.act[m] = m;
        S.rr[m] = B.rr;
        S.stop[m] = B.stop;
        S.alpha[m] = B.alpha;
        S.beta[m] = B.beta;
        S.rrf[m] = B.rr_final;
        S.cit[m] = B.it;
        S.itot[m] = B.it_total;
        S.lastit[m] = B.last_inner;
        S.status[m] = (int)B.status;
        S.mode[m] = I.fresh ? 6 : B.mode;
        S.refs[m] = B.refs;
        S.caps[m] = B.caps;
    }
    __syncthreads();
    batch_split(a, S);
    unsigned epoch = 0;
    const uint64_t pf = l2_evict_first(), pl = l2_evict_last();
    for (int64_t ph = 0; S.nact > 0; ++ph)
    {
        double *const P0 = a.part + (size_t)(2 * (ph & 1)) * kMaxVirt, *const P1 = P0 + kMaxVirt;
        // slices of this block's pieces in a CG phase (opening or iteration), and with PIPE in a
        // refinement's true residual
        auto listed = [](int md) { return md == 0 || md == 3 || md == 6 || (PIPE && md == 2); };
        int T = 0;
        for (int k = 0; k < S.np; ++k)
            if (listed(S.mode[S.act[S.pr_lo + k]]))
                T += S.ps1[k] - S.ps0[k];
        constexpr int kFlatPieces = PIPE ? kPipeFlatPieces : kMaxBatch / 2;
        const bool flat = 2 * T > nw && S.np <= kFlatPieces;
        for (int k = 0; k < S.np; ++k)
        {
            const int r = S.pr_lo + k, m = S.act[r], pidx = S.vs[r] + (int)blockIdx.x - S.fb[r];
            const BInst &I = a.inst[m];
            const int md = S.mode[m];
            double g = 0, d = 0;
            if (md == 1)
            {
                refine_add<float>(I, S.ps0[k], S.ps1[k]);
                continue;
            }
            if (flat && listed(md))
                continue; // dealt below
            if (md == 2)
                g = refine_residual<float>(I, S.ps0[k], S.ps1[k], pf, pl, &d);
            else
            {
                const bool init = md != 0;
                const int cur = (int)(S.cit[m] & 1);
                const float al = (float)S.alpha[m], be = (float)S.beta[m];
                if (I.dim == 2)
                    g = init ? sr_phase<2, true, UV>(I, S.ps0[k], S.ps1[k], 0, md == 6, 0.0f, 0.0f, pf, pl, Un.red, &d)
                             : sr_phase<2, false, UV>(I, S.ps0[k], S.ps1[k], cur, false, al, be, pf, pl, Un.red, &d);
                else
                    g = init ? sr_phase<3, true, UV>(I, S.ps0[k], S.ps1[k], 0, md == 6, 0.0f, 0.0f, pf, pl, Un.red, &d)
                             : sr_phase<3, false, UV>(I, S.ps0[k], S.ps1[k], cur, false, al, be, pf, pl, Un.red, &d);
            }
            block_partial_at(g, P0 + pidx, sh);
            block_partial_at(d, P1 + pidx, sh);
        }
        if (flat)
        {
            // one list of all those slices, dealt round-robin to the warps across the pieces; each
            // warp leaves one (gamma, delta) pair per piece, summed per piece after one block sync
            double *wg = Un.wpart, *wd = Un.wpart + kFlatPieces * 32;
            int off = 0;
            for (int k = 0; k < S.np; ++k)
            {
                const int m = S.act[S.pr_lo + k];
                const int md = S.mode[m];
                if (!listed(md))
                    continue;
                const BInst &I = a.inst[m];
                const int nk = S.ps1[k] - S.ps0[k];
                const int cur = (int)(S.cit[m] & 1);
                const float al = (float)S.alpha[m], be = (float)S.beta[m];
                double lg = 0, ld = 0;
                const int q0 = (warp - off % nw + nw) % nw;
                if constexpr (PIPE)
                {
                    const int s_first = S.ps0[k] + q0, s_end = S.ps1[k];
                    if (md == 2)
                    {
                        // lg, ld: the shares of ||r64||^2 and ||(float) r64||^2
                        if (I.dim == 2)
                            res_slices_pipe<2>(I, s_first, nw, s_end, pf, pl, lg, ld, pipe);
                        else
                            res_slices_pipe<3>(I, s_first, nw, s_end, pf, pl, lg, ld, pipe);
                    }
                    else if (I.dim == 2)
                    {
                        if (md == 0)
                            sr_slices_pipe<2, false>(I, s_first, nw, s_end, cur, false, al, be, pf, pl, lg, ld, pipe);
                        else
                            sr_slices_pipe<2, true>(I, s_first, nw, s_end, 0, md == 6, 0.0f, 0.0f, pf, pl, lg, ld, pipe);
                    }
                    else
                    {
                        if (md == 0)
                            sr_slices_pipe<3, false>(I, s_first, nw, s_end, cur, false, al, be, pf, pl, lg, ld, pipe);
                        else
                            sr_slices_pipe<3, true>(I, s_first, nw, s_end, 0, md == 6, 0.0f, 0.0f, pf, pl, lg, ld, pipe);
                    }
                }
                else
                    for (int q = q0; q < nk; q += nw)
                    {
                        const int sl = S.ps0[k] + q;
                        if (I.dim == 2)
                        {
                            if (md == 0)
                                sr_slice<2, false, UV>(I, sl, cur, false, al, be, pf, pl, lg, ld);
                            else
                                sr_slice<2, true, UV>(I, sl, 0, md == 6, 0.0f, 0.0f, pf, pl, lg, ld);
                        }
                        else
                        {
                            if (md == 0)
                                sr_slice<3, false, UV>(I, sl, cur, false, al, be, pf, pl, lg, ld);
                            else
                                sr_slice<3, true, UV>(I, sl, 0, md == 6, 0.0f, 0.0f, pf, pl, lg, ld);
                        }
                    }
                lg = wsum(lg);
                ld = wsum(ld);
                if (lane == 0)
                {
                    wg[k * 32 + warp] = lg;
                    wd[k * 32 + warp] = ld;
                }
                off += nk;
            }
            __syncthreads();
            for (int k = warp; k < S.np; k += nw)
            {
                const int r = S.pr_lo + k;
                if (!listed(S.mode[S.act[r]]))
                    continue;
                const double tg = wsum(lane < nw ? wg[k * 32 + lane] : 0.0);
                const double td = wsum(lane < nw ? wd[k * 32 + lane] : 0.0);
                if (lane == 0)
                {
                    const int pidx = S.vs[r] + (int)blockIdx.x - S.fb[r];
                    P0[pidx] = tg;
                    P1[pidx] = td;
                }
            }
        }
        if (PIPE && !pipe.ok && lane == 0)
        {
            // a chunk's copy did not complete in time: every block leaves at this barrier
            atomicExch(&a.ctl->fail, 1);
            s_fail = 1;
        }
        if (!batch_barrier(a.ctl, epoch, &s_fail))
            return;
        sr_reduce_decide(a, S, ph, Un.stage);
    }
    if (blockIdx.x == 0)
        for (int m = t; m < a.ninst; m += blockDim.x)
        {
            BState &B = a.st[m];
            B.rr = S.rr[m];
            B.stop = S.stop[m];
            B.alpha = S.alpha[m];
            B.beta = S.beta[m];
            B.rr_final = S.rrf[m];
            B.it = S.cit[m];
            B.it_total = S.itot[m];
            B.last_inner = S.lastit[m];
            B.status = S.status[m];
            B.mode = S.mode[m];
            B.refs = S.refs[m];
            B.caps = S.caps[m];
        }
}

// ---- host side of the batched CG
struct BatchItem
{
    Problem *p;
    bool fp32;
    double rtol, atol, abs_stop;
    int64_t maxit;
    bool fresh;     // false: resume the paused solve whose state is `resume`
    BState resume;
    bool refine;    // FP32 item: the FP64 refinement around it runs in the launch
    double stop64;  // its outer squared-norm target
    int resume_kernel; // FP32 kernel (BatchCtx::launched_sr) that ran the paused solve's last launch
};

// The two FP32 kernel families keep different Krylov states (the single-reduction kernels, 1 and
// 2, keep r, w, s by parity and the Chronopoulos-Gear alpha, beta; the two-reduction kernel, 0,
// keeps p by parity and the textbook alpha, beta), so a paused inner solve resumes only in its own
// family.
inline int fp32_family(int kernel)
{
    return kernel == 0 ? 0 : 1;
}

struct BatchCtx
{
    int device = 0, num_sms = 0, grid = 0;
    int64_t slice = 512; // CG iterations per launch before unfinished solves pause
    size_t smem64 = 0, smem32 = 0; // dynamic shared memory of the two kernel variants
    size_t smem_pipe = 0;          // and of the bulk-copy-fed single-reduction kernel
    int sr = 3; // FP32 inner solves: 1, 2 the single-reduction kernel with 1 or 2 SpMV steps in flight
                // (768 or 512 threads a block); 3 the same with its flat phases fed by bulk copies
                // (384 threads); 0 the two-reduction kernel (LPMGPU_BATCH_SR fixes it)
    // The batch's own tuner of that choice, per launch size: a launch with fewer than kSmallSlices
    // slices per block runs its phases on the column-split path and is bound by the per-iteration
    // floor (barriers, decision passes, one slice's gather chain); a larger one runs the flat
    // path and is bound by the matrix stream, and the best kernel differs between the two.  Unless
    // LPMGPU_BATCH_SR is set, the first kTuneLaunches informative FP32 launches of each size cycle
    // through the kernels and the best serves every later launch of that size.  A large launch is
    // scored by its matrix work (iterations x the members' matrix volume) per second of kernel
    // time; a small one, whose time is its iterations times the floor whatever the members' sizes,
    // by the iterations of its longest solve per second.
    static constexpr int kKernels = 4;
    static constexpr int kTuneLaunches = 3 * kKernels;
    static constexpr int kSmallSlices = 8;
    bool tuning[2] = {false, false};
    static constexpr int kTunePerKernel = kTuneLaunches / kKernels;
    static constexpr double kTuneMinPhases = 64; // shorter launches say little: not counted
    int tune_n[2] = {0, 0}, tune_seen[2] = {0, 0}, pick[2] = {3, 3}, launched_sr = 3, launched_cls = 1;
    double tune_score[2][kKernels][kTunePerKernel] = {};
    double last_ms = 0;

    // Each counted launch scores its kernel (work per kernel second); a kernel's score is the
    // median of its kTunePerKernel launches, robust to one launch that caught an unusual mix.
    void tune_record(double work, double phases)
    {
        const int c = launched_cls;
        if (!tuning[c] || last_ms <= 0)
            return;
        // after three rounds' worth of launches the tuner stops with what it has
        const bool late = ++tune_seen[c] >= 3 * kTuneLaunches;
        if (phases < kTuneMinPhases && !late)
            return;
        if (c == 0)
            work = phases;
        const int v = launched_sr, slot = tune_n[c] / kKernels;
        if (phases >= kTuneMinPhases && slot < kTunePerKernel)
            tune_score[c][v][slot] = work / (last_ms * 1e-3);
        if (++tune_n[c] < kTuneLaunches && !late)
            return;
        double best = -1;
        for (int k = 0; k < kKernels; ++k)
        {
            double sc[kTunePerKernel];
            int m = 0;
            for (int q = 0; q < kTunePerKernel; ++q)
                if (tune_score[c][k][q] > 0)
                    sc[m++] = tune_score[c][k][q];
            if (m == 0)
                continue;
            std::sort(sc, sc + m);
            const double med = sc[m / 2];
            if (std::getenv("LPMGPU_LOG"))
                std::fprintf(stderr, "lpmgpu batch tuner: class %d kernel %d median score %.4g over %d launches\n", c, k,
                             med, m);
            if (med > best)
            {
                best = med;
                pick[c] = k;
            }
        }
        tuning[c] = false;
    }

    cudaStream_t stream = nullptr;
    cudaEvent_t ev_done = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    std::vector<cudaEvent_t> ev_in; // one per item slot
    BInst *d_inst = nullptr, *h_inst = nullptr;
    BState *d_st = nullptr, *h_st = nullptr;
    BCtl *d_ctl = nullptr, *h_ctl = nullptr;
    double *d_part = nullptr;
    int64_t launches = 0;
    double kernel_seconds = 0;
    bool timing_pending = false;

    // grid_cap > 0: at most that many blocks per launch (a lane's share of the SMs)
    cudaError_t init(int dev, int grid_cap = 0)
    {
        device = dev;
        cudaError_t e;
        if ((e = cudaSetDevice(dev)) != cudaSuccess)
            return e;
        if ((e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
            return e;
        smem64 = batch_smem_bytes<double>();
        smem32 = batch_smem_bytes<float>();
        smem_pipe = kSrPipeOffset + (size_t)(kSrPipeThreads / 32) * kPipeWarpBytes;
        {
            const char *env = std::getenv("LPMGPU_BATCH_SR");
            sr = env ? std::atoi(env) : 3;
            if (sr < 0 || sr >= kKernels)
                sr = 3;
            pick[0] = pick[1] = sr;
            tuning[0] = tuning[1] = env == nullptr;
        }
        if ((e = cudaFuncSetAttribute(k_cg_batch_sr<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem32)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(k_cg_batch_sr<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem32)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(k_cg_batch_sr<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem_pipe)) != cudaSuccess)
            return e;
        if ((e = cudaFuncSetAttribute(k_cg_batch<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem64)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(k_cg_batch<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem32)) != cudaSuccess)
            return e;
        int occ64 = 0, occ32 = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, k_cg_batch<double, double>, kBatchThreads<double>,
                                                                smem64)) != cudaSuccess)
            return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, k_cg_batch<float, float>, kBatchThreads<float>,
                                                                smem32)) != cudaSuccess)
            return e;
        int occsr1 = 0, occsr2 = 0, occsr3 = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occsr1, k_cg_batch_sr<1, false>, kSrThreads<1>,
                                                                smem32)) != cudaSuccess ||
            (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occsr2, k_cg_batch_sr<2, false>, kSrThreads<2>,
                                                                smem32)) != cudaSuccess ||
            (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occsr3, k_cg_batch_sr<1, true>, kSrPipeThreads,
                                                                smem_pipe)) != cudaSuccess)
            return e;
        occ32 = std::min({occ32, occsr1, occsr2, occsr3});
        grid = std::min(1024, num_sms * std::max(1, std::min({occ64, occ32, kCGMinBlocks})));
        if (grid_cap > 0)
            grid = std::max(1, std::min(grid, grid_cap));
        if ((e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess)
            return e;
        if ((e = cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming)) != cudaSuccess)
            return e;
        if ((e = cudaEventCreate(&ev_t0)) != cudaSuccess || (e = cudaEventCreate(&ev_t1)) != cudaSuccess)
            return e;
        if ((e = cudaMalloc(&d_inst, sizeof(BInst) * kMaxBatch)) != cudaSuccess ||
            (e = cudaMalloc(&d_st, sizeof(BState) * kMaxBatch)) != cudaSuccess ||
            (e = cudaMalloc(&d_ctl, sizeof(BCtl))) != cudaSuccess ||
            (e = cudaMalloc(&d_part, sizeof(double) * 6 * kMaxVirt)) != cudaSuccess)
            return e;
        if ((e = cudaMallocHost(&h_inst, sizeof(BInst) * kMaxBatch)) != cudaSuccess ||
            (e = cudaMallocHost(&h_st, sizeof(BState) * kMaxBatch)) != cudaSuccess ||
            (e = cudaMallocHost(&h_ctl, sizeof(BCtl))) != cudaSuccess)
            return e;
        return cudaSuccess;
    }

    void release()
    {
        cudaSetDevice(device);
        for (auto ev : ev_in)
            cudaEventDestroy(ev);
        ev_in.clear();
        if (ev_done)
            cudaEventDestroy(ev_done);
        if (ev_t0)
            cudaEventDestroy(ev_t0);
        if (ev_t1)
            cudaEventDestroy(ev_t1);
        if (stream)
            cudaStreamDestroy(stream);
        cudaFree(d_inst);
        cudaFree(d_st);
        cudaFree(d_ctl);
        cudaFree(d_part);
        cudaFreeHost(h_inst);
        cudaFreeHost(h_st);
        cudaFreeHost(h_ctl);
        ev_done = ev_t0 = ev_t1 = nullptr;
        stream = nullptr;
        d_inst = h_inst = nullptr;
        d_st = h_st = nullptr;
        d_ctl = h_ctl = nullptr;
        d_part = nullptr;
    }

    // Enqueues one batched solve after each item's pending work on its own stream; each item's
    // stream then waits for the solve.  Results (h_st, h_ctl) are valid once `stream` is
    // synchronised.  All items must share one precision.
    cudaError_t launch(const std::vector<BatchItem> &items)
    {
        if (items.empty())
            return cudaSuccess;
        if (items.size() > (size_t)kMaxBatch)
            return cudaErrorInvalidValue;
        const int ni = (int)items.size();
        const bool fp32 = items[0].fp32;
        cudaError_t e;
        while ((int)ev_in.size() < ni)
        {
            cudaEvent_t ev;
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
                return e;
            ev_in.push_back(ev);
        }
        for (int m = 0; m < ni; ++m)
        {
            const Problem &p = *items[m].p;
            BInst &I = h_inst[m];
            std::memset(&I, 0, sizeof(I));
            I.dim = p.dim;
            I.fresh = items[m].fresh ? 1 : 0;
            I.n = p.n;
            I.nslices = p.nslices;
            I.ndof = (int64_t)p.n * p.dim;
            I.cost = p.nsb * (p.dim * p.dim + 1);
            I.rowptr = p.cstart;
            I.perm = p.perm;
            I.slice_off = p.slice_off;
            I.col_sell = p.col_sell;
            if (fp32)
            {
                I.K = p.K32;
                I.b = p.b32;
                I.x = p.x32;
                I.r = p.r32;
                I.pa = p.pa32;
                I.pb = p.pb32;
                I.q = p.q32;
                I.r1 = p.r32b;
                I.w1 = p.w32b;
                I.s1 = p.s32b;
            }
            else
            {
                I.K = p.K;
                I.b = p.res;
                I.x = p.x;
                I.r = p.r;
                I.pa = p.p0;
                I.pb = p.p1;
                I.q = p.q;
            }
            I.rtol = items[m].rtol;
            I.atol = items[m].atol;
            I.abs_stop = items[m].abs_stop;
            I.maxit = items[m].maxit;
            I.refine = (fp32 && items[m].refine) ? 1 : 0;
            I.K64 = p.K;
            I.res = p.res;
            I.x64 = p.x;
            I.r64 = p.r;
            I.stop64 = items[m].stop64;
        }
        for (int m = 0; m < ni; ++m)
        {
            if (items[m].fresh)
                std::memset(&h_st[m], 0, sizeof(BState));
            else
            {
                h_st[m] = items[m].resume;
                h_st[m].status &= ~int64_t(8);
            }
        }
        static constexpr int kCand[kKernels] = {3, 1, 2, 0};
        int64_t slices = 0;
        for (int m = 0; m < ni; ++m)
            slices += h_inst[m].nslices;
        const int cls = slices < (int64_t)kSmallSlices * grid ? 0 : 1;
        const int use = (fp32 && tuning[cls]) ? kCand[tune_n[cls] % kKernels] : pick[cls];
        launched_sr = use;
        launched_cls = cls;
        if (fp32)
            for (int m = 0; m < ni; ++m)
            {
                // a paused inner solve of the other kernel family ends here, as if it had met its
                // stop: x64 += x32, the true residual, and a fresh inner solve in this kernel
                BState &B = h_st[m];
                if (items[m].fresh || !items[m].refine || B.mode != 0 ||
                    fp32_family(items[m].resume_kernel) == fp32_family(use))
                    continue;
                B.last_inner = B.it > 0 ? B.it : 1;
                B.refs += 1;
                B.mode = 1;
            }
        std::memset(h_ctl, 0, sizeof(BCtl));
        h_ctl->nact = ni;
        for (int m = 0; m < ni; ++m)
        {
            if ((e = cudaEventRecord(ev_in[m], items[m].p->stream)) != cudaSuccess)
                return e;
            if ((e = cudaStreamWaitEvent(stream, ev_in[m], 0)) != cudaSuccess)
                return e;
        }
        if ((e = cudaMemcpyAsync(d_inst, h_inst, sizeof(BInst) * ni, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_st, h_st, sizeof(BState) * ni, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_ctl, h_ctl, sizeof(BCtl), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return e;
        BArgs a;
        a.inst = d_inst;
        a.st = d_st;
        a.ctl = d_ctl;
        a.part = d_part;
        a.ninst = ni;
        a.slice = slice > 0 ? slice : (int64_t(1) << 62);
        void *args[] = {&a};
        if ((e = cudaEventRecord(ev_t0, stream)) != cudaSuccess)
            return e;
        e = (fp32 && use == 3) ? cudaLaunchCooperativeKernel((const void *)k_cg_batch_sr<1, true>, dim3(grid),
                                                            dim3(kSrPipeThreads), args, smem_pipe, stream)
            : (fp32 && use == 1) ? cudaLaunchCooperativeKernel((const void *)k_cg_batch_sr<1, false>, dim3(grid),
                                                              dim3(kSrThreads<1>), args, smem32, stream)
            : (fp32 && use == 2) ? cudaLaunchCooperativeKernel((const void *)k_cg_batch_sr<2, false>, dim3(grid),
                                                              dim3(kSrThreads<2>), args, smem32, stream)
            : fp32 ? cudaLaunchCooperativeKernel((const void *)k_cg_batch<float, float>, dim3(grid), dim3(kBatchThreads<float>),
                                               args, smem32, stream)
                 : cudaLaunchCooperativeKernel((const void *)k_cg_batch<double, double>, dim3(grid),
                                               dim3(kBatchThreads<double>), args, smem64, stream);
        if (e != cudaSuccess)
            return e;
        if ((e = cudaEventRecord(ev_t1, stream)) != cudaSuccess)
            return e;
        launches++;
        timing_pending = true;
        if ((e = cudaMemcpyAsync(h_st, d_st, sizeof(BState) * ni, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h_ctl, d_ctl, sizeof(BCtl), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
            return e;
        if ((e = cudaEventRecord(ev_done, stream)) != cudaSuccess)
            return e;
        for (int m = 0; m < ni; ++m)
        {
            items[m].p->ctr.kernel_launches++;
            items[m].p->ctr.cg_launches++;
            if ((e = cudaStreamWaitEvent(items[m].p->stream, ev_done, 0)) != cudaSuccess)
                return e;
        }
        return cudaSuccess;
    }

    // after `stream` was synchronised: accumulate the kernel time of the last launch
    void account()
    {
        if (!timing_pending)
            return;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ev_t0, ev_t1) == cudaSuccess)
            kernel_seconds += ms * 1e-3;
        last_ms = ms;
        timing_pending = false;
    }
};

} // namespace lpm

// ======================================================================================
// The batch runtime and its C ABI.
using namespace lpm;

namespace
{

struct StepCopy
{
    std::vector<std::vector<int32_t>> dids, fids;
    std::vector<lpmgpu_dispbc> d;
    std::vector<lpmgpu_forcebc> f;

    explicit StepCopy(const lpmgpu_load_step &s)
    {
        for (int k = 0; k < s.ndisp; ++k)
        {
            dids.emplace_back(s.disp[k].ids, s.disp[k].ids + s.disp[k].count);
            d.push_back(s.disp[k]);
        }
        for (int k = 0; k < s.nforce; ++k)
        {
            fids.emplace_back(s.force[k].ids, s.force[k].ids + s.force[k].count);
            f.push_back(s.force[k]);
        }
        for (size_t k = 0; k < d.size(); ++k)
            d[k].ids = dids[k].data();
        for (size_t k = 0; k < f.size(); ++k)
            f[k].ids = fids[k].data();
    }
};

enum class Ph
{
    Start,       // next sub-step (or next load step) to begin
    NewtonFirst, // force state of the first Newton check in flight
    Newton,      // force state after a Newton update in flight
    NeedCG,      // a CG (FP64, or the FP32 inner solve of a refinement) to start or resume
    DamageCheck, // J2 state + static damage in flight
    Done,
    Failed
};
constexpr int kPhases = 7;

struct Member
{
    lpmgpu_solver *h = nullptr;
    std::vector<StepCopy> steps;
    size_t next = 0;
    std::vector<std::pair<double, int>> stack; // pending sub-steps of the current load step
    double scale = 1.0;
    int depth = 0;
    Ph ph = Ph::Start;
    bool pending = false; // device work whose scalars the next synchronisation delivers
    int k = 0;
    double tol_mult = 0, nres = 0;
    lpmgpu_stats cur{};
    std::vector<lpmgpu_stats> step_stats;
    lpmgpu_stats total{};
    int64_t dof_iters = 0;
    int32_t status = LPMGPU_OK;
    std::chrono::steady_clock::time_point t_add, t_done;
    // the CG in progress (it may span several launches) and the mixed-precision refinement
    bool ls_fresh = true;
    BState ls_state{};
    int ls_kernel = 1; // the FP32 kernel of the paused solve's last launch
    double ir_stop = 0, ir_rr = 0;
    // fatigue members (SolverFatigue, include/solver_fatigue.h): steps [0, nstatic) run as
    // solveProblemStatic's steps, the rest as cycle steps; cycle_end[s] = (closes a cycle, dN/dt)
    bool fatigue = false;
    size_t nstatic = 0;
    std::vector<std::pair<bool, double>> cycle_end;
    // the lane that solves this member's linear systems, and the member's weight in its balance
    int lane = 0;
    int64_t cost = 0;
    // solo: the member's linear solves run alone through the single-problem CG (solo_solves)
    bool solo = false;
    int64_t lane_cost() const { return solo ? 0 : cost; }
};

// A lane: a share of the SMs with its own batched CG launches (FP64 members, then the FP32 inner
// solves of mixed members, one launch of each in flight at most; the FP32 launch waits for the
// FP64 one so the lane never holds more than its share).  Lanes progress independently: while
// one lane's members take their host decisions and run their per-member kernels, the other
// lanes' CG kernels keep the GPU busy, and a lane's short solves wait only for its own long
// ones.  The lanes' shares add up to at most one block per SM, so every launch in flight can
// be resident at once, as its grid barrier needs.
struct Lane
{
    BatchCtx c64, c32;
    bool inflight = false;
    std::vector<Member *> g64, g32; // members of the launches in flight
    int64_t cost = 0;               // summed matrix cost of its live members
    int64_t launches = 0;
};

int32_t cuda_status(cudaError_t e, const char *what)
{
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? LPMGPU_ERR_OUT_OF_MEMORY : LPMGPU_ERR_CUDA;
}

} // namespace

struct lpmgpu_batch
{
    int device = 0;
    int64_t slice = 512;
    int64_t solo_bytes = kDefaultSoloBytes;
    std::vector<std::unique_ptr<Lane>> lanes;
    std::vector<std::unique_ptr<Member>> members; // index = member id; removed -> null
    lpmgpu_batch_stats stats{};
    std::chrono::steady_clock::time_point t_create;
    int64_t round_max_it = 0; // most CG iterations one member ran in this round's launches

    Problem &P(Member &m) { return m.h->p; }

    // one sub-step begins: scaled load step (solver_static.h:78-87 halving), assembly, first
    // force state of the Newton loop.  Returns false when the member has finished its path.
    int32_t begin_substep(Member &m)
    {
        if (m.stack.empty())
        {
            if (m.next >= m.steps.size())
            {
                finish(m, LPMGPU_OK);
                return LPMGPU_OK;
            }
            m.stack.push_back({1.0, 0});
            m.next++;
            m.cur = lpmgpu_stats{};
        }
        auto sd = m.stack.back();
        m.stack.pop_back();
        m.scale = sd.first;
        m.depth = sd.second;
        const StepCopy &s = m.steps[m.next - 1];
        std::vector<lpmgpu_dispbc> db(s.d);
        std::vector<lpmgpu_forcebc> fb(s.f);
        for (auto &d : db)
            d.step *= m.scale;
        for (auto &f : fb)
        {
            f.fx *= m.scale;
            f.fy *= m.scale;
            f.fz *= m.scale;
        }
        lpmgpu_load_step ls{db.data(), (int32_t)db.size(), fb.data(), (int32_t)fb.size()};
        Problem &p = P(m);
        cudaError_t e = launch_apply_bc(p, ls);
        if (e == cudaSuccess && !p.desc.tangent) // tangent mode assembles before every solve
            e = enqueue_assemble(p, true);
        if (e == cudaSuccess)
            e = enqueue_force_state(p, true);
        if (e != cudaSuccess)
            return fail_member(m, cuda_status(e, "batch sub-step"));
        m.cur.damage_iters++;
        m.ph = Ph::NewtonFirst;
        m.pending = true;
        return LPMGPU_OK;
    }

    int32_t fail_member(Member &m, int32_t code)
    {
        m.status = code;
        m.ph = Ph::Failed;
        m.pending = false;
        m.t_done = std::chrono::steady_clock::now();
        stats.members_failed++;
        lanes[m.lane]->cost -= m.lane_cost();
        return LPMGPU_OK;
    }

    void finish(Member &m, int32_t code)
    {
        m.status = code;
        m.ph = Ph::Done;
        m.pending = false;
        m.t_done = std::chrono::steady_clock::now();
        stats.members_done++;
        lanes[m.lane]->cost -= m.lane_cost();
    }

    double kernel_seconds() const
    {
        double t = 0;
        for (auto &L : lanes)
            t += L->c64.kernel_seconds + L->c32.kernel_seconds;
        return t;
    }

    // (Re)creates the lanes; only while no member is running.  The SMs are split evenly.
    cudaError_t make_lanes(int nl)
    {
        for (auto &L : lanes)
        {
            L->c64.release();
            L->c32.release();
        }
        lanes.clear();
        int sms = 0;
        cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess)
            return e;
        nl = std::max(1, std::min(nl, std::max(1, sms / 8)));
        for (int l = 0; l < nl; ++l)
        {
            auto L = std::make_unique<Lane>();
            const int cap = (nl == 1) ? 0 : sms / nl;
            if ((e = L->c64.init(device, cap)) != cudaSuccess || (e = L->c32.init(device, cap)) != cudaSuccess)
            {
                L->c64.release();
                L->c32.release();
                return e;
            }
            L->c64.slice = L->c32.slice = slice;
            lanes.push_back(std::move(L));
        }
        return cudaSuccess;
    }

    void release()
    {
        for (auto &L : lanes)
        {
            L->c64.release();
            L->c32.release();
        }
        lanes.clear();
    }

    // after the Newton loop of a fatigue member's step (SolverFatigue::solveProblemStep has no
    // damage loop, solver_fatigue.h:278-302).  A static step (solveProblemStatic, :244-275) that
    // failed is reset and halved, and a converged one is followed by updateStateVar and
    // storeStateVar.  A cycle step (solveProblemOneCycle, :221-241) is followed by updateStateVar
    // whether it converged or not; the cycle's last step adds updateFatigueDamage(dN/dt),
    // storeStateVar, updateGeometry and updateForceState.
    int32_t after_newton_fatigue(Member &m, int n_newton)
    {
        Problem &p = P(m);
        const size_t si = m.next - 1;
        const bool is_static = si < m.nstatic, failed = n_newton >= p.desc.max_iter;
        if (is_static && failed)
            return fail_substep(m);
        cudaError_t e = launch_update_state_var(p);
        if (e == cudaSuccess && is_static)
            e = enqueue_store_state(p);
        if (e == cudaSuccess && !is_static)
        {
            if (failed)
                m.cur.cuts++; // a cycle step whose Newton failed, carried on from
            if (m.cycle_end[si].first)
            {
                e = launch_fatigue_damage(p, m.cycle_end[si].second);
                if (e == cudaSuccess)
                    e = enqueue_store_state(p);
                if (e == cudaSuccess)
                    e = enqueue_force_state(p, false);
            }
        }
        if (e != cudaSuccess)
            return fail_member(m, cuda_status(e, "batch fatigue step"));
        substep_done(m);
        return LPMGPU_OK;
    }

    // after the Newton loop of one damage iteration (solver_static.h:119-121)
    int32_t after_newton(Member &m, int n_newton)
    {
        Problem &p = P(m);
        m.cur.residual_norm = m.nres;
        if (m.fatigue)
            return after_newton_fatigue(m, n_newton);
        if (n_newton >= p.desc.max_iter)
            return fail_substep(m);
        cudaError_t e = enqueue_damage_update(p);
        if (e != cudaSuccess)
            return fail_member(m, cuda_status(e, "batch damage update"));
        m.ph = Ph::DamageCheck;
        m.pending = true;
        return LPMGPU_OK;
    }

    // Newton failure: reset to the last converged state and run two halves (solver_static.h:78-87)
    int32_t fail_substep(Member &m)
    {
        if (m.depth >= 30)
            return fail_member(m, LPMGPU_ERR_CUTS);
        cudaError_t e = enqueue_reset_state(P(m));
        if (e != cudaSuccess)
            return fail_member(m, cuda_status(e, "batch reset"));
        m.cur.cuts++;
        m.stack.push_back({m.scale / 2.0, m.depth + 1});
        m.stack.push_back({m.scale / 2.0, m.depth + 1});
        m.ph = Ph::Start;
        return LPMGPU_OK;
    }

    void substep_done(Member &m)
    {
        Problem &p = P(m);
        m.cur.reaction_norm = std::sqrt(p.scal_host->reaction_sq);
        if (m.stack.empty())
        {
            m.cur.converged = 1;
            m.step_stats.push_back(m.cur);
            m.total.converged = 1;
            m.total.newton_solves += m.cur.newton_solves;
            m.total.cuts += m.cur.cuts;
            m.total.damage_iters += m.cur.damage_iters;
            m.total.cg_iters += m.cur.cg_iters;
            m.total.cg_maxit_hits += m.cur.cg_maxit_hits;
            m.total.refinements += m.cur.refinements;
            m.total.reaction_norm = m.cur.reaction_norm;
            m.total.residual_norm = m.cur.residual_norm;
            if (m.next >= m.steps.size())
            {
                finish(m, LPMGPU_OK);
                return;
            }
        }
        m.ph = Ph::Start;
    }

    // Solver::NewtonIteration's test (solver.h:55-90) after a force state arrived
    int32_t newton_check(Member &m)
    {
        Problem &p = P(m);
        if (m.nres <= p.desc.tol_iter * m.tol_mult)
            return after_newton(m, m.k);
        if (++m.k > p.desc.max_iter)
            return after_newton(m, p.desc.max_iter);
        return start_linear(m);
    }

    // one linear solve K x = res: FP64 CG, or (mixed) FP32 inner CGs inside an FP64 refinement
    // on the same squared-norm rule (the loop of solve_dim in cg.cu).  With x = 0 the first true
    // residual is res itself, whose squared norm the force state just delivered (updateRR), so
    // the first inner solve starts at once from b32 = (float) res.
    int32_t start_linear(Member &m)
    {
        Problem &p = P(m);
        m.cur.newton_solves++;
        m.ls_fresh = true;
        if (p.desc.tangent)
        {
            // tangent mode: K (and its FP32 copy) from the current state before every solve
            const cudaError_t e0 = enqueue_assemble(p, true);
            if (e0 != cudaSuccess)
                return fail_member(m, cuda_status(e0, "batch tangent assembly"));
        }
        if (p.desc.precision != LPMGPU_MIXED || m.solo)
        {
            m.ph = Ph::NeedCG; // a solo member's solve sets up its own refinement
            return LPMGPU_OK;
        }
        m.ir_rr = p.scal_host->res_sq;
        m.ir_stop = p.desc.cg_rtol * m.ir_rr + p.desc.cg_atol;
        cudaError_t e = cudaMemsetAsync(p.x, 0, sizeof(double) * (size_t)p.n * p.dim, p.stream);
        if (e != cudaSuccess)
            return fail_member(m, cuda_status(e, "batched refinement"));
        if (m.ir_rr <= m.ir_stop)
            return finish_linear(m);
        if ((e = enqueue_res_to_b32(p)) != cudaSuccess)
            return fail_member(m, cuda_status(e, "batched refinement"));
        m.ph = Ph::NeedCG;
        return LPMGPU_OK;
    }

    // Newton update with the solution and the next force state
    int32_t finish_linear(Member &m)
    {
        Problem &p = P(m);
        cudaError_t e = launch_add_disp(p);
        if (e == cudaSuccess)
            e = enqueue_force_state(p, true);
        if (e != cudaSuccess)
            return fail_member(m, cuda_status(e, "batch Newton update"));
        m.ph = Ph::Newton;
        m.pending = true;
        return LPMGPU_OK;
    }

    int32_t resolve(Member &m)
    {
        Problem &p = P(m);
        m.pending = false;
        if (p.scal_host->err)
            return fail_member(m, LPMGPU_ERR_TOPOLOGY);
        switch (m.ph)
        {
        case Ph::NewtonFirst:
        {
            m.nres = std::sqrt(p.scal_host->res_sq);
            const double nreac = std::sqrt(p.scal_host->reaction_sq);
            m.tol_mult = std_max(m.nres, nreac);
            m.k = 0;
            return newton_check(m);
        }
        case Ph::Newton:
            m.nres = std::sqrt(p.scal_host->res_sq);
            return newton_check(m);
        case Ph::DamageCheck:
        {
            const bool new_damaged = p.scal_host->any_flag != 0;
            cudaError_t e = enqueue_store_state(p);
            if (e == cudaSuccess && new_damaged)
            {
                // damage loop (solver_static.h:126-139): force state, then assemble + Newton again
                e = enqueue_force_state(p, false);
                if (e == cudaSuccess && !p.desc.tangent)
                    e = enqueue_assemble(p, true);
                if (e == cudaSuccess)
                    e = enqueue_force_state(p, true);
                if (e == cudaSuccess)
                {
                    m.cur.damage_iters++;
                    m.ph = Ph::NewtonFirst;
                    m.pending = true;
                    return LPMGPU_OK;
                }
            }
            if (e != cudaSuccess)
                return fail_member(m, cuda_status(e, "batch damage loop"));
            substep_done(m);
            return LPMGPU_OK;
        }
        default:
            return LPMGPU_OK;
        }
    }

    cudaError_t sync_members(const std::vector<Member *> &ms)
    {
        for (Member *m : ms)
        {
            cudaError_t e = cudaStreamSynchronize(P(*m).stream);
            if (e != cudaSuccess)
                return e;
        }
        return cudaSuccess;
    }

    // Enqueues one batched launch over members of one precision that need a CG (fresh solves and
    // solves paused by an earlier launch's iteration slice), without waiting for it.
    int32_t launch_group(BatchCtx &ctx, std::vector<Member *> &ms, bool fp32)
    {
        if (ms.empty())
            return LPMGPU_OK;
        std::vector<BatchItem> items;
        for (Member *m : ms)
        {
            Problem &p = P(*m);
            const int64_t ndof = (int64_t)p.n * p.dim;
            BatchItem it{&p,           fp32,
                         fp32 ? 0.0 : p.desc.cg_rtol,
                         fp32 ? 0.0 : p.desc.cg_atol,
                         fp32 ? 0.25 * m->ir_stop : -1.0,
                         p.desc.cg_maxit > 0 ? p.desc.cg_maxit : ndof,
                         m->ls_fresh,  m->ls_state,
                         fp32,         m->ir_stop,
                         m->ls_kernel};
            items.push_back(it);
        }
        cudaError_t e = ctx.launch(items);
        if (e != cudaSuccess)
            return cuda_status(e, "batched CG launch");
        stats.cg_launches++;
        return LPMGPU_OK;
    }

    // After the launch of `ctx` finished: each member's CG state, and the follow-up work of the
    // solves that ended.
    int32_t finish_group(BatchCtx &ctx, std::vector<Member *> &ms, bool fp32)
    {
        if (ms.empty())
            return LPMGPU_OK;
        cudaError_t e;
        if ((e = cudaStreamSynchronize(ctx.stream)) != cudaSuccess)
            return cuda_status(e, "batched CG");
        ctx.account();
        const bool timeout = ctx.h_ctl->fail != 0;
        double work = 0;
        int64_t phases = 0;
        for (size_t q = 0; q < ms.size(); ++q)
        {
            const int64_t before = ms[q]->ls_fresh ? 0 : ms[q]->ls_state.it_total;
            work += (double)(ctx.h_st[q].it_total - before) * (double)ms[q]->cost;
            phases = std::max(phases, ctx.h_st[q].it_total - before);
        }
        if (fp32 && !timeout)
            ctx.tune_record(work, (double)phases);
        for (size_t q = 0; q < ms.size(); ++q)
        {
            Member &m = *ms[q];
            Problem &p = P(m);
            const BState &S = ctx.h_st[q];
            const int64_t before = m.ls_fresh ? 0 : m.ls_state.it_total;
            const int64_t done_now = S.it_total - before;
            round_max_it = std::max(round_max_it, done_now);
            m.cur.cg_iters += done_now;
            m.dof_iters += done_now * (int64_t)p.n * p.dim;
            p.ctr.cg_iters += done_now;
            m.ls_state = S;
            m.ls_kernel = ctx.launched_sr;
            if (timeout)
            {
                set_last_error("a device-side barrier wait timed out in the batched CG kernel");
                fail_member(m, LPMGPU_ERR_TIMEOUT);
                continue;
            }
            if (S.status & 8)
            {
                m.ls_fresh = false; // paused: resumes in the lane's next launch
                continue;
            }
            if (fp32)
            {
                // the FP64 refinement ran to its end inside the launch (solve_dim's loop)
                m.cur.refinements += S.refs;
                m.cur.cg_maxit_hits += S.caps;
            }
            else if (S.status & 1)
                m.cur.cg_maxit_hits++;
            finish_linear(m);
        }
        ms.clear();
        return LPMGPU_OK;
    }

    // The linear solves of the solo members waiting for one, each through the single-problem
    // persistent CG (solve_linear: FP64, or FP32 inner solves in FP64 refinement, on the
    // problem's own stream), one at a time with no batched launch in flight, so that every
    // cooperative launch has the GPU to itself; then each one's Newton update is enqueued.
    int32_t solo_solves(bool *ran)
    {
        *ran = false;
        bool any = false;
        for (auto &up : members)
            if (up && up->solo && up->ph == Ph::NeedCG)
                any = true;
        if (!any)
            return LPMGPU_OK;
        for (auto &L : lanes)
            if (L->inflight)
            {
                const int32_t r = complete_lane(*L);
                if (r != LPMGPU_OK)
                    return r;
            }
        for (auto &up : members)
        {
            if (!up || !up->solo || up->ph != Ph::NeedCG)
                continue;
            Member &m = *up;
            Problem &p = P(m);
            cudaSetDevice(p.device);
            CGResult r;
            const cudaError_t e = solve_linear(p, r);
            *ran = true;
            stats.solo_solves++;
            if (e != cudaSuccess)
            {
                fail_member(m, cuda_status(e, "solo linear solve"));
                continue;
            }
            if (r.timeout)
            {
                set_last_error("a device-side barrier wait timed out in the CG kernel");
                fail_member(m, LPMGPU_ERR_TIMEOUT);
                continue;
            }
            m.cur.cg_iters += r.iters;
            m.cur.cg_maxit_hits += r.maxit_hits;
            m.cur.refinements += r.refinements;
            m.dof_iters += r.iters * (int64_t)p.n * p.dim;
            round_max_it = std::max(round_max_it, r.iters);
            finish_linear(m);
        }
        return LPMGPU_OK;
    }

    // A lane's launches: the FP64 members waiting for a CG, then the FP32 inner solves of its
    // mixed members (at most kMaxBatch of each per launch; the rest wait for the next one).
    int32_t launch_lane(int l)
    {
        Lane &L = *lanes[l];
        L.g64.clear();
        L.g32.clear();
        for (auto &up : members)
            if (up && up->lane == l && up->ph == Ph::NeedCG && !up->solo)
            {
                auto &g = P(*up).desc.precision == LPMGPU_MIXED ? L.g32 : L.g64;
                if ((int)g.size() < kMaxBatch)
                    g.push_back(up.get());
            }
        if (L.g64.empty() && L.g32.empty())
            return LPMGPU_OK;
        int32_t r = launch_group(L.c64, L.g64, false);
        if (r != LPMGPU_OK)
            return r;
        if (!L.g64.empty() && !L.g32.empty())
        {
            // the FP32 launch starts after the FP64 one: the lane never holds more than its share
            const cudaError_t e = cudaStreamWaitEvent(L.c32.stream, L.c64.ev_done, 0);
            if (e != cudaSuccess)
                return cuda_status(e, "batched CG launch");
        }
        if ((r = launch_group(L.c32, L.g32, true)) != LPMGPU_OK)
            return r;
        L.inflight = true;
        L.launches++;
        return LPMGPU_OK;
    }

    bool lane_ready(Lane &L)
    {
        const cudaEvent_t ev = !L.g32.empty() ? L.c32.ev_done : L.c64.ev_done;
        return cudaEventQuery(ev) == cudaSuccess;
    }

    int32_t complete_lane(Lane &L)
    {
        int32_t r = finish_group(L.c64, L.g64, false);
        if (r == LPMGPU_OK)
            r = finish_group(L.c32, L.g32, true);
        L.inflight = false;
        return r;
    }

    // The host passes of one lane's members: until each waits for a CG (or is finished), start
    // sub-steps, wait once for all their pending scalars, take their decisions, repeat.
    int32_t host_passes(int l)
    {
        for (int pass = 0; pass < 1000; ++pass)
        {
            for (auto &up : members)
                if (up && up->lane == l && up->ph == Ph::Start)
                {
                    cudaSetDevice(P(*up).device);
                    begin_substep(*up);
                }
            std::vector<Member *> pend;
            for (auto &up : members)
                if (up && up->lane == l && up->pending)
                    pend.push_back(up.get());
            if (pend.empty())
                break;
            cudaError_t e = sync_members(pend);
            if (e != cudaSuccess)
                return cuda_status(e, "batch round");
            for (Member *m : pend)
                resolve(*m);
        }
        return LPMGPU_OK;
    }

    // One round: every lane whose launches finished takes its members' results; every idle
    // lane runs its members' host passes and starts its next launch.  When no lane could do
    // anything, the round waits for the lane launched first.  With one lane this is the loop of
    // one launch for all members followed by their host decisions.
    int32_t round(int32_t *running)
    {
        static const bool log = std::getenv("LPMGPU_LOG") != nullptr;
        const auto t_round = std::chrono::steady_clock::now();
        const double k0 = kernel_seconds();
        const int64_t l0 = stats.cg_launches;
        round_max_it = 0;
        stats.rounds++;
        bool progressed = false;
        for (auto &L : lanes)
            if (L->inflight && lane_ready(*L))
            {
                const int32_t r = complete_lane(*L);
                if (r != LPMGPU_OK)
                    return r;
                progressed = true;
            }
        double solo_ms = 0;
        {
            const auto t_solo = std::chrono::steady_clock::now();
            bool ran = false;
            const int32_t r = solo_solves(&ran);
            if (r != LPMGPU_OK)
                return r;
            progressed = progressed || ran;
            solo_ms = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_solo).count() * 1e3;
        }
        int launched = 0;
        for (int l = 0; l < (int)lanes.size(); ++l)
        {
            if (lanes[l]->inflight)
                continue;
            int32_t r = host_passes(l);
            if (r == LPMGPU_OK)
                r = launch_lane(l);
            if (r != LPMGPU_OK)
                return r;
            if (lanes[l]->inflight)
                launched++;
        }
        if (!progressed && launched == 0)
        {
            // nothing finished and nothing new to start: wait for the lane in flight longest
            Lane *oldest = nullptr;
            for (auto &L : lanes)
                if (L->inflight && (!oldest || L->launches < oldest->launches))
                    oldest = L.get();
            if (oldest)
            {
                int32_t r = complete_lane(*oldest);
                const int l = (int)(std::find_if(lanes.begin(), lanes.end(),
                                                 [&](const std::unique_ptr<Lane> &x) { return x.get() == oldest; }) -
                                    lanes.begin());
                if (r == LPMGPU_OK)
                    r = host_passes(l);
                if (r == LPMGPU_OK)
                    r = launch_lane(l);
                if (r != LPMGPU_OK)
                    return r;
            }
        }
        int32_t live = 0;
        for (auto &up : members)
            if (up && up->ph != Ph::Done && up->ph != Ph::Failed)
                live++;
        if (running)
            *running = live;
        if (live == 0)
            for (auto &L : lanes)
                if (L->inflight)
                {
                    const int32_t r = complete_lane(*L);
                    if (r != LPMGPU_OK)
                        return r;
                }
        if (log)
        {
            int nph[kPhases] = {0};
            for (auto &up : members)
                if (up)
                    nph[(int)up->ph]++;
            int infl = 0;
            for (auto &L : lanes)
                infl += L->inflight ? 1 : 0;
            std::fprintf(stderr,
                         "lpmgpu batch round %lld: lanes in flight %d/%zu launches=%lld max_it=%lld kernel_ms=%.3f "
                         "round_ms=%.3f solo_ms=%.3f phases(start,nf,n,cg,dmg,done,fail)=%d,%d,%d,%d,%d,%d,%d\n",
                         (long long)stats.rounds, infl, lanes.size(), (long long)(stats.cg_launches - l0),
                         (long long)round_max_it, (kernel_seconds() - k0) * 1e3,
                         std::chrono::duration<double>(std::chrono::steady_clock::now() - t_round).count() * 1e3,
                         solo_ms, nph[0], nph[1], nph[2], nph[3], nph[4], nph[5], nph[6]);
        }
        return LPMGPU_OK;
    }
};

extern "C" {

int32_t lpmgpu_batch_create(int32_t device, lpmgpu_batch **out)
{
    if (!out)
        return LPMGPU_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    {
        set_last_error("no CUDA device visible; liblpmgpu has no CPU path");
        return LPMGPU_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev)
        return LPMGPU_ERR_INVALID_ARG;
    auto *b = new lpmgpu_batch();
    b->device = device;
    const char *env = std::getenv("LPMGPU_BATCH_LANES");
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess)
        e = b->make_lanes(env ? std::max(1, std::atoi(env)) : kDefaultLanes);
    if (e != cudaSuccess)
    {
        int32_t s = cuda_status(e, "lpmgpu_batch_create");
        b->release();
        delete b;
        return s;
    }
    b->t_create = std::chrono::steady_clock::now();
    *out = b;
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_destroy(lpmgpu_batch *b)
{
    if (!b)
        return LPMGPU_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    for (auto &L : b->lanes)
        if (L->inflight)
            b->complete_lane(*L);
    b->release();
    delete b;
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_set_lanes(lpmgpu_batch *b, int32_t lanes)
{
    if (!b || lanes < 1)
        return LPMGPU_ERR_INVALID_ARG;
    for (auto &up : b->members)
        if (up && up->ph != Ph::Done && up->ph != Ph::Failed)
        {
            set_last_error("the lanes of a batch can change only while no member is running");
            return LPMGPU_ERR_NOT_READY;
        }
    if (cudaSetDevice(b->device) != cudaSuccess)
        return LPMGPU_ERR_CUDA;
    const cudaError_t e = b->make_lanes(lanes);
    if (e != cudaSuccess)
        return cuda_status(e, "lpmgpu_batch_set_lanes");
    return LPMGPU_OK;
}

// Checks a problem that is to join the batch; LPMGPU_OK when it may.
static int32_t check_joiner(lpmgpu_batch *b, lpmgpu_solver *h)
{
    if (h->p.device != b->device)
    {
        set_last_error("the problem lives on another device than the batch");
        return LPMGPU_ERR_INVALID_ARG;
    }
    if (h->p.desc.direct == 1)
    {
        set_last_error("the batch solves its members by the batched CG; a problem with desc.direct = 1 cannot join");
        return LPMGPU_ERR_INVALID_ARG;
    }
    int live = 0;
    for (auto &up : b->members)
    {
        if (up && up->h == h && up->ph != Ph::Done && up->ph != Ph::Failed)
        {
            set_last_error("the problem is already a running member of this batch");
            return LPMGPU_ERR_INVALID_ARG;
        }
        if (up && up->ph != Ph::Done && up->ph != Ph::Failed)
            live++;
    }
    if (live >= kMaxMembers)
    {
        set_last_error("a batch runs at most 4096 problems at once");
        return LPMGPU_ERR_BUDGET;
    }
    return LPMGPU_OK;
}

static int32_t push_member(lpmgpu_batch *b, std::unique_ptr<Member> m, int32_t *member)
{
    m->t_add = std::chrono::steady_clock::now();
    // the lane with the least matrix volume among its running members
    const Problem &p = m->h->p;
    m->cost = p.nsb * (p.dim * p.dim + 1);
    m->solo = b->solo_bytes > 0 && cg_stream_bytes(p) >= b->solo_bytes;
    int best = 0;
    for (int l = 1; l < (int)b->lanes.size(); ++l)
        if (b->lanes[l]->cost < b->lanes[best]->cost)
            best = l;
    m->lane = best;
    b->lanes[best]->cost += m->lane_cost();
    if (m->steps.empty())
    {
        m->ph = Ph::Done;
        m->t_done = m->t_add;
        b->stats.members_done++;
        b->lanes[best]->cost -= m->lane_cost();
    }
    b->members.push_back(std::move(m));
    if (member)
        *member = (int32_t)b->members.size() - 1;
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_add(lpmgpu_batch *b, lpmgpu_solver *h, const lpmgpu_load_step *steps, int32_t nsteps,
                         int32_t *member)
{
    if (!b || !h || nsteps < 0 || (nsteps > 0 && !steps))
        return LPMGPU_ERR_INVALID_ARG;
    const int32_t c = check_joiner(b, h);
    if (c != LPMGPU_OK)
        return c;
    for (int32_t s = 0; s < nsteps; ++s)
        for (int k = 0; k < steps[s].ndisp; ++k)
            if (steps[s].disp[k].flag < 0 || steps[s].disp[k].flag >= h->p.dim || steps[s].disp[k].count < 0 ||
                (steps[s].disp[k].count > 0 && !steps[s].disp[k].ids))
                return LPMGPU_ERR_INVALID_ARG;
    auto m = std::make_unique<Member>();
    m->h = h;
    for (int32_t s = 0; s < nsteps; ++s)
        m->steps.emplace_back(steps[s]);
    return push_member(b, std::move(m), member);
}

int32_t lpmgpu_batch_add_fatigue(lpmgpu_batch *b, lpmgpu_solver *h, const lpmgpu_load_step *static_steps,
                                 int32_t nstatic, const lpmgpu_load_step *cycle_steps, int32_t cycle_len,
                                 int32_t ncycles, const double *dndt, int32_t *member)
{
    if (!b || !h || nstatic < 0 || (nstatic > 0 && !static_steps) || cycle_len < 0 || ncycles < 0 ||
        (ncycles > 0 && (cycle_len == 0 || !cycle_steps || !dndt)))
        return LPMGPU_ERR_INVALID_ARG;
    const int32_t c = check_joiner(b, h);
    if (c != LPMGPU_OK)
        return c;
    auto check = [&](const lpmgpu_load_step &st) {
        for (int k = 0; k < st.ndisp; ++k)
            if (st.disp[k].flag < 0 || st.disp[k].flag > 2 || st.disp[k].count < 0 ||
                (st.disp[k].count > 0 && !st.disp[k].ids))
                return false;
        for (int k = 0; k < st.nforce; ++k)
            if (st.force[k].count < 0 || (st.force[k].count > 0 && !st.force[k].ids))
                return false;
        return true;
    };
    const int64_t ncs = (int64_t)cycle_len * ncycles;
    for (int32_t s = 0; s < nstatic; ++s)
        if (!check(static_steps[s]))
            return LPMGPU_ERR_INVALID_ARG;
    for (int64_t s = 0; s < ncs; ++s)
        if (!check(cycle_steps[s]))
            return LPMGPU_ERR_INVALID_ARG;
    auto m = std::make_unique<Member>();
    m->h = h;
    m->fatigue = true;
    m->nstatic = (size_t)nstatic;
    for (int32_t s = 0; s < nstatic; ++s)
    {
        m->steps.emplace_back(static_steps[s]);
        m->cycle_end.push_back({false, 0.0});
    }
    for (int64_t s = 0; s < ncs; ++s)
    {
        m->steps.emplace_back(cycle_steps[s]);
        const bool end = (s + 1) % cycle_len == 0;
        m->cycle_end.push_back({end, end ? dndt[s / cycle_len] : 0.0});
    }
    return push_member(b, std::move(m), member);
}

int32_t lpmgpu_batch_round(lpmgpu_batch *b, int32_t *running)
{
    if (!b)
        return LPMGPU_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess)
        return LPMGPU_ERR_CUDA;
    return b->round(running);
}

int32_t lpmgpu_batch_run(lpmgpu_batch *b)
{
    if (!b)
        return LPMGPU_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess)
        return LPMGPU_ERR_CUDA;
    const auto t0 = std::chrono::steady_clock::now();
    int32_t running = 1;
    while (running > 0)
    {
        int32_t r = b->round(&running);
        if (r != LPMGPU_OK)
            return r;
    }
    b->stats.seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_member(const lpmgpu_batch *b, int32_t member, lpmgpu_member_info *info)
{
    if (!b || !info || member < 0 || member >= (int32_t)b->members.size() || !b->members[member])
        return LPMGPU_ERR_INVALID_ARG;
    const Member &m = *b->members[member];
    std::memset(info, 0, sizeof(*info));
    info->state = m.ph == Ph::Done ? 1 : (m.ph == Ph::Failed ? 2 : 0);
    info->status = m.status;
    info->steps_done = (int32_t)m.step_stats.size();
    info->nsteps = (int32_t)m.steps.size();
    info->total = m.total;
    info->dof_iters = m.dof_iters;
    const auto end = (info->state != 0) ? m.t_done : std::chrono::steady_clock::now();
    info->seconds = std::chrono::duration<double>(end - m.t_add).count();
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_member_steps(const lpmgpu_batch *b, int32_t member, lpmgpu_stats *steps, int32_t cap,
                                  int32_t *count)
{
    if (!b || member < 0 || member >= (int32_t)b->members.size() || !b->members[member] || cap < 0 ||
        (cap > 0 && !steps))
        return LPMGPU_ERR_INVALID_ARG;
    const Member &m = *b->members[member];
    const int32_t n = (int32_t)m.step_stats.size();
    for (int32_t k = 0; k < std::min(n, cap); ++k)
        steps[k] = m.step_stats[k];
    if (count)
        *count = n;
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_remove(lpmgpu_batch *b, int32_t member)
{
    if (!b || member < 0 || member >= (int32_t)b->members.size() || !b->members[member])
        return LPMGPU_ERR_INVALID_ARG;
    const Member &m = *b->members[member];
    if (m.ph != Ph::Done && m.ph != Ph::Failed)
    {
        set_last_error("only finished members can be removed");
        return LPMGPU_ERR_NOT_READY;
    }
    b->members[member].reset();
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_set_slice(lpmgpu_batch *b, int64_t iterations)
{
    if (!b || iterations < 0)
        return LPMGPU_ERR_INVALID_ARG;
    b->slice = iterations;
    for (auto &L : b->lanes)
        L->c64.slice = L->c32.slice = iterations;
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_set_solo_bytes(lpmgpu_batch *b, int64_t bytes)
{
    if (!b || bytes < 0)
        return LPMGPU_ERR_INVALID_ARG;
    b->solo_bytes = bytes;
    return LPMGPU_OK;
}

int32_t lpmgpu_batch_get_stats(const lpmgpu_batch *b, lpmgpu_batch_stats *st)
{
    if (!b || !st)
        return LPMGPU_ERR_INVALID_ARG;
    *st = b->stats;
    st->cg_kernel_seconds = b->kernel_seconds();
    st->fp32_kernel = b->lanes.empty() ? -1 : b->lanes[0]->c32.pick[1];
    st->fp32_kernel_small = b->lanes.empty() ? -1 : b->lanes[0]->c32.pick[0];
    st->fp32_tuning = (!b->lanes.empty() && (b->lanes[0]->c32.tuning[0] || b->lanes[0]->c32.tuning[1])) ? 1 : 0;
    int64_t it = 0, di = 0;
    for (auto &up : b->members)
        if (up)
        {
            it += up->total.cg_iters;
            di += up->dof_iters;
        }
    st->cg_iters = it;
    st->dof_iters = di;
    return LPMGPU_OK;
}

} // extern "C"
