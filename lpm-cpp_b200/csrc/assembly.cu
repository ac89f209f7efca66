// Global stiffness assembly: one CTA per particle row, deterministic, no atomics.  The
// output is the sliced-ELL layout described in lpm_internal.cuh.
//
// The reference (include/stiffness.h:198-361) evaluates localStiffnessANA(pi, pj) for every
// pj in conns(pi) by re-walking bond lists (include/derivative.h:8-239), then scatters
// 0.5*K(i,j) into row block i and 0.5*K(i,j)^T into row block j, so the stored upper block is
// 0.5*K(i,j) + 0.5*K(j,i)^T.  Here the CTA owning row i computes both K(i,j) and K(j,i) for
// each j in conns(i) and writes the final symmetric block once, into a full block-CSR.
//
// The local blocks are restated as sums over bond paths of one layer L:
//   K_L(i,j) = [j in N_L(i)] (direct(i->j) - sum_{k != j} other(i->j, i->k))
//              - sum_{k in N_L(i), j in N_L(k)} hop(i->k, k->j)
// with the terms accumulated in exactly the order derivative.h visits them (bond lists are
// ascending in partner id, so "for k in N_L(i)" and "for k in N_L(j)" agree on common
// neighbours), each expression rounded as the reference rounds it.  With -fmad=false the
// blocks are bit-identical to the reference's.
//
// The displacement-BC elimination (stiffness.h:364-438) is folded into the write: every entry
// in the row or column of a constrained DOF (disp BC or damage_visual == 1) is zeroed, and
// the constrained diagonal entries are set to ||diag(K)|| by a second kernel.
#include "lpm_internal.cuh"

namespace lpm
{



struct AsmArgs
{
    int n, mb, mrec;
    const int *__restrict__ bstart, *__restrict__ nb0, *__restrict__ bp2, *__restrict__ brev;
    const int *__restrict__ cstart, *__restrict__ conns, *__restrict__ cons;
    const int *__restrict__ perm;
    const int64_t *__restrict__ slice_off;
    const double *__restrict__ cs, *__restrict__ Kn, *__restrict__ Tv, *__restrict__ bdamage;
    const double *__restrict__ cs_sum, *__restrict__ damage_visual;
    double *__restrict__ K, *__restrict__ diag_raw;
    int apply_bc;
};

// Shared-memory staging of particle i's neighbourhood.  Own bonds a (i -> k) keep their full
// record; every same-layer bond of every neighbour k (k -> x) is a "record" holding its cosines,
// T = (1 - D) Tv (the product the reference forms inline, same rounding), its partner x, the
// slot of x in conns(i), and the cosines and T of the opposite bond x -> k.
struct AsmSmem
{
    double *o_cs, *o_Kn, *o_Tv, *o_D, *o_S; // own bonds [mb*3], [mb], [mb], [mb], [mb*3] (S of k)
    double *o_rKn, *o_rTv, *o_rD;            // the opposite bond k -> i of own bond a
    double *n_cs, *n_T, *r_cs, *r_T;          // records [mrec*3], [mrec], [mrec*3], [mrec]
    int *conns;                               // [kMaxConns]
    int *o_p2, *o_revpos, *o_L, *n_off;       // [mb], [mb], [mb], [mb+1]
    int *n_p2, *n_slot;                       // [mrec]
    signed char *dir, *hop;                   // [2][kMaxConns], [mb][kMaxConns]
};

__host__ __device__ inline size_t asm_smem_bytes(int mb, int mrec)
{
    return sizeof(double) * (12 * (size_t)mb + 8 * (size_t)mrec) +
           sizeof(int) * (kMaxConns + 4 * (size_t)mb + 1 + 2 * (size_t)mrec) +
           sizeof(signed char) * ((2 + (size_t)mb) * kMaxConns) + 64;
}

__device__ inline AsmSmem carve(void *base, int mb, int mrec)
{
    AsmSmem s;
    double *d = static_cast<double *>(base);
    s.o_cs = d;
    d += 3 * mb;
    s.o_Kn = d;
    d += mb;
    s.o_Tv = d;
    d += mb;
    s.o_D = d;
    d += mb;
    s.o_S = d;
    d += 3 * mb;
    s.o_rKn = d;
    d += mb;
    s.o_rTv = d;
    d += mb;
    s.o_rD = d;
    d += mb;
    s.n_cs = d;
    d += 3 * mrec;
    s.n_T = d;
    d += mrec;
    s.r_cs = d;
    d += 3 * mrec;
    s.r_T = d;
    d += mrec;
    int *q = reinterpret_cast<int *>(d);
    s.conns = q;
    q += kMaxConns;
    s.o_p2 = q;
    q += mb;
    s.o_revpos = q;
    q += mb;
    s.o_L = q;
    q += mb;
    s.n_off = q;
    q += mb + 1;
    s.n_p2 = q;
    q += mrec;
    s.n_slot = q;
    q += mrec;
    signed char *c = reinterpret_cast<signed char *>(q);
    s.dir = c;
    c += 2 * kMaxConns;
    s.hop = c;
    return s;
}

__device__ __forceinline__ int find_slot(const int *conns, int nc, int x)
{
    int lo = 0, hi = nc - 1;
    while (lo <= hi)
    {
        const int mid = (lo + hi) >> 1;
        const int v = conns[mid];
        if (v == x)
            return mid;
        if (v < x)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return -1;
}

// Row R of K(i, j) (fr[c] = K(i,j)[R][c]) and column R of K(j, i) (gc[c] = K(j,i)[c][R]) receive,
// entry by entry, the operations derivative.h applies:
//   other bond (derivative.h:91-99):  -= 0.5*((1-D1)Tv1 + (1-D2)Tv2) * cs2[row] * cs1[col]
//   two-hop    (derivative.h:105-113, 128-136): -= 0.5*(T_B + T_A) * csA[row] * csB[col]
//   direct     (derivative.h:62-87):  += (1-D)((-Kn cs[col] + Tv S_j[col]) cs[row] - (Kn+Tv) cs.cs)
// where (Kn+Tv) cs.cs is (Kn+Tv)*(cs[r]*cs[r]) on the diagonal (pow(cs,2)) and
// (Kn+Tv)*cs[hi]*cs[lo] off it (coordinate order x < y < z), as the reference writes them.
template <int D>
__device__ __forceinline__ void sub_other_row(double fr[D], int R, double T1, const double *c1, double T2,
                                              const double *c2)
{
    const double t = 0.5 * (T1 + T2);
#pragma unroll
    for (int c = 0; c < D; ++c)
        fr[c] -= t * c2[R] * c1[c];
}
template <int D>
__device__ __forceinline__ void sub_other_col(double gc[D], int R, double T1, const double *c1, double T2,
                                              const double *c2)
{
    const double t = 0.5 * (T1 + T2);
#pragma unroll
    for (int c = 0; c < D; ++c)
        gc[c] -= t * c2[c] * c1[R];
}
template <int D>
__device__ __forceinline__ void sub_hop_row(double fr[D], int R, double TA, const double *cA, double TB,
                                            const double *cB)
{
    const double t = 0.5 * (TB + TA);
#pragma unroll
    for (int c = 0; c < D; ++c)
        fr[c] -= t * cA[R] * cB[c];
}
template <int D>
__device__ __forceinline__ void sub_hop_col(double gc[D], int R, double TA, const double *cA, double TB,
                                            const double *cB)
{
    const double t = 0.5 * (TB + TA);
#pragma unroll
    for (int c = 0; c < D; ++c)
        gc[c] -= t * cA[c] * cB[R];
}
// (Kn+Tv) cs_r cs_q in the reference's operator order
__device__ __forceinline__ double pkt_rt(double kt, const double *c, int r, int q)
{
    if (r == q)
        return kt * (c[r] * c[r]);
    return kt * c[r > q ? r : q] * c[r > q ? q : r];
}
template <int D>
__device__ __forceinline__ void add_direct_row(double fr[D], int R, double Dm, double Kn, double Tv, const double *c,
                                               const double *S)
{
    const double kt = Kn + Tv;
#pragma unroll
    for (int q = 0; q < D; ++q)
        fr[q] += (1 - Dm) * ((-Kn * c[q] + Tv * S[q]) * c[R] - pkt_rt(kt, c, R, q));
}
template <int D>
__device__ __forceinline__ void add_direct_col(double gc[D], int R, double Dm, double Kn, double Tv, const double *c,
                                               const double *S)
{
    const double kt = Kn + Tv;
#pragma unroll
    for (int r = 0; r < D; ++r)
        gc[r] += (1 - Dm) * ((-Kn * c[R] + Tv * S[R]) * c[r] - pkt_rt(kt, c, r, R));
}

// All D rows of K_L(i, j) (f[R][c]) and of K_L(j, i)^T (g[R][c], column R in j's orientation)
// for slot sl, layer L, in one walk over the layer's bond paths.  Each entry receives its updates
// in the order derivative.h applies them.
template <int D, int L>
__device__ __forceinline__ void layer_all(const AsmSmem &s, int sl, int olo, int ohi, const double *Si, double f[D][D],
                                          double g[D][D])
{
    const int aj = s.dir[L * kMaxConns + sl];
    for (int o = olo; o < ohi; ++o)
    {
        const double *co = s.o_cs + 3 * o;
        const double To = (1 - s.o_D[o]) * s.o_Tv[o];
        const int hb = s.hop[o * kMaxConns + sl];
        if (aj >= 0)
        {
            if (o == aj)
            {
#pragma unroll
                for (int R = 0; R < D; ++R)
                    add_direct_row<D>(f[R], R, s.o_D[o], s.o_Kn[o], s.o_Tv[o], co, s.o_S + 3 * o);
                continue;
            }
            const double Taj = (1 - s.o_D[aj]) * s.o_Tv[aj];
#pragma unroll
            for (int R = 0; R < D; ++R)
                sub_other_row<D>(f[R], R, Taj, s.o_cs + 3 * aj, To, co);
        }
        if (hb >= 0)
        {
            const int q = s.n_off[o] + hb;
#pragma unroll
            for (int R = 0; R < D; ++R)
                sub_hop_row<D>(f[R], R, To, co, s.n_T[q], s.n_cs + 3 * q);
        }
    }
    if (aj >= 0)
    {
        const int jlo = s.n_off[aj], jhi = s.n_off[aj + 1];
        const int rji = jlo + s.o_revpos[aj];
        const double Tji = s.n_T[rji];
        const double *cji = s.n_cs + 3 * rji;
        for (int q = jlo; q < jhi; ++q)
        {
            const double *cq = s.n_cs + 3 * q;
            if (q == rji)
            {
#pragma unroll
                for (int R = 0; R < D; ++R)
                    add_direct_col<D>(g[R], R, s.o_rD[aj], s.o_rKn[aj], s.o_rTv[aj], cq, Si);
                continue;
            }
#pragma unroll
            for (int R = 0; R < D; ++R)
                sub_other_col<D>(g[R], R, Tji, cji, s.n_T[q], cq);
            const int xs = s.n_slot[q];
            const int ax = (xs >= 0) ? s.dir[L * kMaxConns + xs] : -1;
            if (ax >= 0)
            {
                const int rxi = s.n_off[ax] + s.o_revpos[ax];
#pragma unroll
                for (int R = 0; R < D; ++R)
                    sub_hop_col<D>(g[R], R, s.n_T[q], cq, s.n_T[rxi], s.n_cs + 3 * rxi);
            }
        }
    }
    else
    {
        for (int o = olo; o < ohi; ++o)
        {
            const int hb = s.hop[o * kMaxConns + sl];
            if (hb < 0)
                continue;
            const int q = s.n_off[o] + hb;
            const int rki = s.n_off[o] + s.o_revpos[o];
#pragma unroll
            for (int R = 0; R < D; ++R)
                sub_hop_col<D>(g[R], R, s.r_T[q], s.r_cs + 3 * q, s.n_T[rki], s.n_cs + 3 * rki);
        }
    }
}

template <int D>
__global__ void __launch_bounds__(256) k_assemble(AsmArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // CTAs run in sliced-ELL order, so the rows of one slice (whose entries interleave in
    // memory) are written at about the same time and their partial sectors merge in L2
    const int pos = blockIdx.x;
    const int i = a.perm[pos];
    const int lane = pos % kSlice;
    const int64_t sbase = a.slice_off[pos / kSlice];
    const int tid = threadIdx.x;
    AsmSmem s = carve(smem_raw, a.mb, a.mrec);

    const int b0 = a.bstart[i], nbi = a.bstart[i + 1] - b0, n0 = a.nb0[i];
    const int c0 = a.cstart[i], nc = a.cstart[i + 1] - c0;
    for (int q = tid; q < nc; q += blockDim.x)
        s.conns[q] = a.conns[c0 + q];
    {
        // dir and hop are adjacent byte tables ((2 + nbi) x kMaxConns, word aligned): -1 everywhere
        int *w = reinterpret_cast<int *>(s.dir);
        const int nw = (2 + nbi) * kMaxConns / 4;
        for (int q = tid; q < nw; q += blockDim.x)
            w[q] = -1;
    }
    for (int o = tid; o < nbi; o += blockDim.x)
    {
        const int b = b0 + o, k = a.bp2[b], L = (o < n0) ? 0 : 1;
        const int klo = (L == 0) ? a.bstart[k] : a.bstart[k] + a.nb0[k];
        const int khi = (L == 0) ? a.bstart[k] + a.nb0[k] : a.bstart[k + 1];
        const int rb = a.brev[b];
        s.o_p2[o] = k;
        s.o_L[o] = L;
        s.o_revpos[o] = rb - klo;
        s.n_off[o + 1] = khi - klo; // counts, scanned below
        for (int c = 0; c < 3; ++c)
        {
            s.o_cs[3 * o + c] = a.cs[3 * (int64_t)b + c];
            s.o_S[3 * o + c] = a.cs_sum[6 * (int64_t)k + 3 * L + c];
        }
        s.o_Kn[o] = a.Kn[b];
        s.o_Tv[o] = a.Tv[b];
        s.o_D[o] = a.bdamage[b];
        s.o_rKn[o] = a.Kn[rb];
        s.o_rTv[o] = a.Tv[rb];
        s.o_rD[o] = a.bdamage[rb];
    }
    __syncthreads();
    if (tid == 0)
    {
        s.n_off[0] = 0;
        for (int o = 0; o < nbi; ++o)
            s.n_off[o + 1] += s.n_off[o];
    }
    __syncthreads();
    const int ntot = s.n_off[nbi];
    for (int q = tid; q < ntot; q += blockDim.x)
    {
        int o = 0;
        while (s.n_off[o + 1] <= q)
            ++o;
        const int k = s.o_p2[o], L = s.o_L[o];
        const int klo = (L == 0) ? a.bstart[k] : a.bstart[k] + a.nb0[k];
        const int b = klo + (q - s.n_off[o]);
        const int x = a.bp2[b];
        const int rb = a.brev[b];
        s.n_p2[q] = x;
        const int sl = find_slot(s.conns, nc, x);
        s.n_slot[q] = sl;
        for (int c = 0; c < 3; ++c)
        {
            s.n_cs[3 * q + c] = a.cs[3 * (int64_t)b + c];
            s.r_cs[3 * q + c] = a.cs[3 * (int64_t)rb + c];
        }
        s.n_T[q] = (1 - a.bdamage[b]) * a.Tv[b];
        s.r_T[q] = (1 - a.bdamage[rb]) * a.Tv[rb];
        if (sl >= 0)
            s.hop[o * kMaxConns + sl] = (signed char)(q - s.n_off[o]);
    }
    for (int o = tid; o < nbi; o += blockDim.x)
    {
        const int sl = find_slot(s.conns, nc, s.o_p2[o]);
        if (sl >= 0)
            s.dir[s.o_L[o] * kMaxConns + sl] = (signed char)o;
    }
    __syncthreads();

    const int selfslot = find_slot(s.conns, nc, i);
    const double dvi = a.damage_visual[i];
    bool ci[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        ci[k] = a.apply_bc && (k < D) && (a.cons[3 * i + k] == 1 || fabs(dvi - 1.0) < kEps);
    const double *Si0 = a.cs_sum + 6 * (int64_t)i, *Si1 = Si0 + 3;

    // one thread per connection slot: all D rows of block (i, conns[sl])
    for (int sl = tid; sl < nc; sl += blockDim.x)
    {
        const int j = s.conns[sl];
        double out[D][D];
        if (sl == selfslot)
        {
            // fdu2dxyz (derivative.h:8-45): one accumulator over both layers; row R of the upper
            // part is acc[R][q >= R], the mirrored entries come from the rows above
            double acc[D][D];
#pragma unroll
            for (int R = 0; R < D; ++R)
#pragma unroll
                for (int q = 0; q < D; ++q)
                    acc[R][q] = 0.0;
            for (int o = 0; o < nbi; ++o)
            {
                const double *c = s.o_cs + 3 * o;
                const double Dm = s.o_D[o], Kn = s.o_Kn[o], Tv = s.o_Tv[o], kt = Kn + Tv;
                const double *S = (s.o_L[o] == 0) ? Si0 : Si1;
#pragma unroll
                for (int R = 0; R < D; ++R)
#pragma unroll
                    for (int q = 0; q < D; ++q)
                    {
                        // entry (min(R,q), max(R,q)) of the upper triangle
                        const int rr = R < q ? R : q, cc = R < q ? q : R;
                        acc[R][q] += (1 - Dm) * ((Kn * c[cc] + Tv * S[cc]) * c[rr] + pkt_rt(kt, c, rr, cc));
                    }
            }
#pragma unroll
            for (int R = 0; R < D; ++R)
            {
#pragma unroll
                for (int q = 0; q < D; ++q)
                    out[R][q] = acc[R][q];
                a.diag_raw[(int64_t)D * i + R] = out[R][R];
#pragma unroll
                for (int q = 0; q < D; ++q)
                    if (R != q && (ci[R] || ci[q]))
                        out[R][q] = 0.0;
            }
        }
        else
        {
            double f0[D][D], f1[D][D], g0[D][D], g1[D][D];
#pragma unroll
            for (int R = 0; R < D; ++R)
#pragma unroll
                for (int q = 0; q < D; ++q)
                {
                    f0[R][q] = 0.0;
                    f1[R][q] = 0.0;
                    g0[R][q] = 0.0;
                    g1[R][q] = 0.0;
                }
            layer_all<D, 0>(s, sl, 0, n0, Si0, f0, g0);
            layer_all<D, 1>(s, sl, n0, nbi, Si1, f1, g1);
            const double dvj = a.damage_visual[j];
            bool cj[D];
#pragma unroll
            for (int q = 0; q < D; ++q)
                cj[q] = a.apply_bc && (a.cons[3 * j + q] == 1 || fabs(dvj - 1.0) < kEps);
#pragma unroll
            for (int R = 0; R < D; ++R)
#pragma unroll
                for (int q = 0; q < D; ++q)
                {
                    const double kij = f0[R][q] + f1[R][q];
                    const double kji = g0[R][q] + g1[R][q];
                    const double v = 0.5 * kij + 0.5 * kji;
                    out[R][q] = (ci[R] || cj[q]) ? 0.0 : v;
                }
        }
        double *dst = a.K + (sbase + sl) * D * D * kSlice + lane;
#pragma unroll
        for (int R = 0; R < D; ++R)
#pragma unroll
            for (int q = 0; q < D; ++q)
                dst[(R * D + q) * kSlice] = out[R][q];
    }
}

__device__ __forceinline__ double warp_sum_d(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// norm_diag = ||diag(K)||_2 before the elimination (stiffness.h:368-378), fixed-order tree
__global__ void k_diag_norm(int64_t m, const double *__restrict__ diag, Scalars *scal)
{
    __shared__ double sh[32];
    double v = 0;
    for (int64_t q = threadIdx.x; q < m; q += blockDim.x)
        v += diag[q] * diag[q];
    v = warp_sum_d(v);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        double r = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : 0.0;
        r = warp_sum_d(r);
        if (threadIdx.x == 0)
            scal->norm_diag = sqrt(r);
    }
}

// the self block is connection slot nconn - nconn_largeq (conns >= i are the last nlq entries)
__global__ void k_bc_diag(int n, int dim, const int *__restrict__ perm, const int64_t *__restrict__ slice_off,
                          const int *__restrict__ cstart, const int *__restrict__ nlq, const int *__restrict__ cons,
                          const double *__restrict__ damage_visual, const Scalars *__restrict__ scal,
                          double *__restrict__ K, float *__restrict__ K32, double *__restrict__ res)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n)
        return;
    const int i = perm[pos];
    const bool dmg = fabs(damage_visual[i] - 1.0) < kEps;
    const int self = (cstart[i + 1] - cstart[i]) - nlq[i];
    const int64_t b = slice_off[pos / kSlice] + self;
    const double nd = scal->norm_diag;
    for (int k = 0; k < dim; ++k)
        if (cons[3 * i + k] == 1 || dmg)
        {
            K[(b * dim * dim + k * dim + k) * kSlice + pos % kSlice] = nd;
            if (K32)
                K32[(b * dim * dim + k * dim + k) * kSlice + pos % kSlice] = (float)nd;
            res[(int64_t)dim * i + k] = 0.0; // updateStiffnessDispBC zeroes the residual (stiffness.h:434)
        }
}

cudaError_t launch_assemble(Problem &p, bool apply_bc, bool *k32_written)
{
    cudaError_t e;
    if (k32_written)
        *k32_written = false;
    if (p.asm_fast && !p.asm_exact)
    {
        // the fast form writes the FP32 copy too when the caller wants one
        const bool k32 = k32_written != nullptr && p.K32 != nullptr;
        if ((e = launch_assemble_fast(p, apply_bc, k32)) != cudaSuccess)
            return e;
        if (apply_bc)
        {
            k_diag_norm<<<1, 1024, 0, p.stream>>>((int64_t)p.n * p.dim, p.diag_raw, p.scal);
            k_bc_diag<<<div_up(p.n, 256), 256, 0, p.stream>>>(p.n, p.dim, p.perm, p.slice_off, p.cstart, p.nlq,
                                                              p.cons, p.damage_visual, p.scal, p.K,
                                                              k32 ? p.K32 : nullptr, p.res);
            p.ctr.kernel_launches += 2;
            if ((e = cudaGetLastError()) != cudaSuccess)
                return e;
        }
        if (k32_written)
            *k32_written = k32;
        return cudaSuccess;
    }
    AsmArgs a;
    a.n = p.n;
    a.mb = p.max_bonds;
    a.mrec = p.max_records;
    a.bstart = p.bstart;
    a.nb0 = p.nb0;
    a.bp2 = p.bp2;
    a.brev = p.brev;
    a.cstart = p.cstart;
    a.conns = p.conns;
    a.cons = p.cons;
    a.cs = p.cs;
    a.Kn = p.Kn;
    a.Tv = p.Tv;
    a.bdamage = p.bdamage;
    a.cs_sum = p.cs_sum;
    a.damage_visual = p.damage_visual;
    a.perm = p.perm;
    a.slice_off = p.slice_off;
    a.K = p.K;
    a.diag_raw = p.diag_raw;
    a.apply_bc = apply_bc ? 1 : 0;
    const size_t smem = asm_smem_bytes(a.mb, a.mrec);
    // one thread per connection slot (more threads per block cost more in occupancy than they
    // gain in the staging: measured 3.5 ms vs 5.0 ms per SC 20 mm assembly at 128)
    const int threads = std::min(256, std::max(32, ((p.max_conns + 31) / 32) * 32));
    if (p.dim == 2)
    {
        if ((e = cudaFuncSetAttribute(k_assemble<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
            return e;
        k_assemble<2><<<p.n, threads, smem, p.stream>>>(a);
    }
    else
    {
        if ((e = cudaFuncSetAttribute(k_assemble<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
            return e;
        k_assemble<3><<<p.n, threads, smem, p.stream>>>(a);
    }
    p.ctr.kernel_launches++;
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    if (apply_bc)
    {
        k_diag_norm<<<1, 1024, 0, p.stream>>>((int64_t)p.n * p.dim, p.diag_raw, p.scal);
        k_bc_diag<<<div_up(p.n, 256), 256, 0, p.stream>>>(p.n, p.dim, p.perm, p.slice_off, p.cstart, p.nlq, p.cons,
                                                          p.damage_visual, p.scal, p.K, nullptr, p.res);
        p.ctr.kernel_launches += 2;
        e = cudaGetLastError();
    }
    return e;
}

// Reference layout (stiffness.h:24-26, 198-361): row (i, r) starts at
// K_pointer[i] + r*dim*nlq - r(r-1)/2; self block entries c >= r, then the blocks of conns >= i.
__global__ void k_export_ref(int n, int dim, const int *__restrict__ cstart, const int *__restrict__ conns,
                             const int *__restrict__ nlq, const int64_t *__restrict__ kp, const int *__restrict__ iperm,
                             const int64_t *__restrict__ slice_off, const double *__restrict__ K,
                             int64_t *__restrict__ IK, int64_t *__restrict__ JK, double *__restrict__ V)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * dim)
        return;
    const int i = t / dim, r = t % dim;
    const int c0 = cstart[i], nc = cstart[i + 1] - c0, m = nlq[i];
    const int self = nc - m;
    const int pos = iperm[i], lane = pos % kSlice;
    const int64_t sbase = slice_off[pos / kSlice];
    const int64_t start = kp[i] + (int64_t)r * dim * m - (int64_t)r * (r - 1) / 2;
    IK[(int64_t)dim * i + r] = start + 1;
    int64_t out = start;
    for (int num = 0; num < m; ++num)
    {
        const int sl = self + num, j = conns[c0 + sl];
        const double *blk = K + (sbase + sl) * dim * dim * kSlice + lane;
        for (int c = (num == 0 ? r : 0); c < dim; ++c)
        {
            JK[out] = (int64_t)dim * j + c + 1;
            V[out] = blk[(r * dim + c) * kSlice];
            out++;
        }
    }
    if (t == 0)
        IK[(int64_t)dim * n] = kp[n] + 1;
}

cudaError_t launch_export_ref(const Problem &p, int64_t *IK, int64_t *JK, double *K)
{
    k_export_ref<<<div_up((int64_t)p.n * p.dim, 256), 256, 0, p.stream>>>(p.n, p.dim, p.cstart, p.conns, p.nlq,
                                                                          p.kp_ref, p.iperm, p.slice_off, p.K, IK, JK, K);
    return cudaGetLastError();
}

} // namespace lpm
