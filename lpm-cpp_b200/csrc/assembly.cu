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

constexpr int kAsmThreads = 64;

struct AsmArgs
{
    int n, dim, mb;
    const int *__restrict__ bstart, *__restrict__ nb0, *__restrict__ bp2, *__restrict__ brev;
    const int *__restrict__ cstart, *__restrict__ conns, *__restrict__ cons;
    const int *__restrict__ perm;
    const int64_t *__restrict__ slice_off;
    const double *__restrict__ cs, *__restrict__ Kn, *__restrict__ Tv, *__restrict__ bdamage;
    const double *__restrict__ cs_sum, *__restrict__ damage_visual;
    double *__restrict__ K, *__restrict__ diag_raw;
    int apply_bc;
};

// shared-memory staging of particle i's neighbourhood
struct AsmSmem
{
    int *conns;                      // [kMaxConns]
    int *o_p2, *o_revpos, *o_L, *n_off; // own bonds [mb], n_off [mb+1]
    double *o_cs, *o_Kn, *o_Tv, *o_D, *o_S; // [mb*3], [mb], [mb], [mb], [mb*3]
    int *n_p2, *n_slot, *n_rev;      // neighbour (same-layer) bonds [mb*mb]
    double *n_cs, *n_Kn, *n_Tv, *n_D; // [mb*mb*3], [mb*mb] ...
    signed char *dir;                // [2][kMaxConns]
    signed char *hop;                // [mb][kMaxConns]
};

__host__ __device__ inline size_t asm_smem_bytes(int mb)
{
    const size_t m2 = (size_t)mb * mb;
    return sizeof(int) * (kMaxConns + 4 * (size_t)mb + 1 + 3 * m2) +
           sizeof(double) * (3 * (size_t)mb + 3 * (size_t)mb + 3 * (size_t)mb + 3 * m2 + 3 * m2) +
           sizeof(signed char) * ((2 + (size_t)mb) * kMaxConns) + 64;
}

__device__ inline AsmSmem carve(void *base, int mb)
{
    AsmSmem s;
    const size_t m2 = (size_t)mb * mb;
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
    s.n_cs = d;
    d += 3 * m2;
    s.n_Kn = d;
    d += m2;
    s.n_Tv = d;
    d += m2;
    s.n_D = d;
    d += m2;
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
    q += m2;
    s.n_slot = q;
    q += m2;
    s.n_rev = q;
    q += m2;
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

// (Kn+Tv) * cs_r * cs_c as the reference writes it: pow(cs, 2) on the diagonal,
// cs_hi * cs_lo (coordinate order x < y < z) off the diagonal (derivative.h:17-33, 62-87)
__device__ __forceinline__ double pkt(double kt, const double *c, int r, int q)
{
    if (r == q)
        return kt * (c[r] * c[r]);
    const int hi = r > q ? r : q, lo = r > q ? q : r;
    return kt * c[hi] * c[lo];
}

// the "other bond" term of derivative.h:91-99: bond 1 gives the column cosine, bond 2 the row
__device__ __forceinline__ void sub_other(double acc[3][3], int d, double D1, double Tv1, const double *c1, double D2,
                                          double Tv2, const double *c2)
{
    const double t = 0.5 * ((1 - D1) * Tv1 + (1 - D2) * Tv2);
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c)
            acc[r][c] -= t * c2[r] * c1[c];
}

// the two-hop term i->k (bond A), k->j (bond B) of derivative.h:105-113 / 128-136
__device__ __forceinline__ void sub_hop(double acc[3][3], int d, double DA, double TvA, const double *cA, double DB,
                                        double TvB, const double *cB)
{
    const double t = 0.5 * ((1 - DB) * TvB + (1 - DA) * TvA);
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c)
            acc[r][c] -= t * cA[r] * cB[c];
}

// the direct term of derivative.h:62-87: bond i->j with the cosine sum S of particle j
__device__ __forceinline__ void add_direct(double acc[3][3], int d, double D, double Kn, double Tv, const double *c,
                                           const double *S)
{
    const double kt = Kn + Tv;
    for (int r = 0; r < d; ++r)
        for (int q = 0; q < d; ++q)
            acc[r][q] += (1 - D) * ((-Kn * c[q] + Tv * S[q]) * c[r] - pkt(kt, c, r, q));
}

__global__ void __launch_bounds__(kAsmThreads) k_assemble(AsmArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // CTAs run in sliced-ELL order, so the rows of one slice (whose entries interleave in
    // memory) are written at about the same time and their partial sectors merge in L2
    const int pos = blockIdx.x;
    const int i = a.perm[pos];
    const int lane = pos % kSlice;
    const int64_t sbase = a.slice_off[pos / kSlice];
    const int tid = threadIdx.x;
    const int mb = a.mb, d = a.dim;
    AsmSmem s = carve(smem_raw, mb);

    const int b0 = a.bstart[i], nbi = a.bstart[i + 1] - b0, n0 = a.nb0[i];
    const int c0 = a.cstart[i], nc = a.cstart[i + 1] - c0;
    for (int q = tid; q < nc; q += kAsmThreads)
        s.conns[q] = a.conns[c0 + q];
    for (int q = tid; q < 2 * kMaxConns; q += kAsmThreads)
        s.dir[q] = -1;
    for (int q = tid; q < nbi * kMaxConns; q += kAsmThreads)
        s.hop[q] = -1;
    // own bonds
    for (int o = tid; o < nbi; o += kAsmThreads)
    {
        const int b = b0 + o, k = a.bp2[b], L = (o < n0) ? 0 : 1;
        const int klo = (L == 0) ? a.bstart[k] : a.bstart[k] + a.nb0[k];
        const int khi = (L == 0) ? a.bstart[k] + a.nb0[k] : a.bstart[k + 1];
        s.o_p2[o] = k;
        s.o_L[o] = L;
        s.o_revpos[o] = a.brev[b] - klo;
        s.n_off[o + 1] = khi - klo; // counts, scanned below
        for (int c = 0; c < 3; ++c)
        {
            s.o_cs[3 * o + c] = a.cs[3 * (int64_t)b + c];
            s.o_S[3 * o + c] = a.cs_sum[6 * (int64_t)k + 3 * L + c];
        }
        s.o_Kn[o] = a.Kn[b];
        s.o_Tv[o] = a.Tv[b];
        s.o_D[o] = a.bdamage[b];
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
    // neighbours' same-layer bonds
    for (int q = tid; q < ntot; q += kAsmThreads)
    {
        int o = 0;
        while (s.n_off[o + 1] <= q)
            ++o;
        const int k = s.o_p2[o], L = s.o_L[o];
        const int klo = (L == 0) ? a.bstart[k] : a.bstart[k] + a.nb0[k];
        const int b = klo + (q - s.n_off[o]);
        const int x = a.bp2[b];
        s.n_p2[q] = x;
        s.n_rev[q] = a.brev[b];
        s.n_slot[q] = find_slot(s.conns, nc, x);
        for (int c = 0; c < 3; ++c)
            s.n_cs[3 * q + c] = a.cs[3 * (int64_t)b + c];
        s.n_Kn[q] = a.Kn[b];
        s.n_Tv[q] = a.Tv[b];
        s.n_D[q] = a.bdamage[b];
    }
    __syncthreads();
    for (int o = tid; o < nbi; o += kAsmThreads)
    {
        const int sl = find_slot(s.conns, nc, s.o_p2[o]);
        if (sl >= 0)
            s.dir[s.o_L[o] * kMaxConns + sl] = (signed char)o;
    }
    for (int q = tid; q < ntot; q += kAsmThreads)
    {
        int o = 0;
        while (s.n_off[o + 1] <= q)
            ++o;
        const int sl = s.n_slot[q];
        if (sl >= 0)
            s.hop[o * kMaxConns + sl] = (signed char)(q - s.n_off[o]);
    }
    __syncthreads();

    const int selfslot = find_slot(s.conns, nc, i);
    const double dvi = a.damage_visual[i];
    bool ci[3];
    for (int k = 0; k < 3; ++k)
        ci[k] = a.apply_bc && (k < d) && (a.cons[3 * i + k] == 1 || fabs(dvi - 1.0) < kEps);

    for (int sl = tid; sl < nc; sl += kAsmThreads)
    {
        const int j = s.conns[sl];
        double out[3][3];
        if (sl == selfslot)
        {
            // fdu2dxyz (derivative.h:8-45): one accumulator over both layers, upper part
            double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int o = 0; o < nbi; ++o)
            {
                const int L = s.o_L[o];
                const double *c = s.o_cs + 3 * o;
                const double D = s.o_D[o], Kn = s.o_Kn[o], Tv = s.o_Tv[o], kt = Kn + Tv;
                const double *S = a.cs_sum + 6 * (int64_t)i + 3 * L;
                for (int r = 0; r < d; ++r)
                    for (int q = r; q < d; ++q)
                        acc[r][q] += (1 - D) * ((Kn * c[q] + Tv * S[q]) * c[r] + pkt(kt, c, r, q));
            }
            for (int r = 0; r < d; ++r)
                for (int q = 0; q < d; ++q)
                    out[r][q] = (q >= r) ? acc[r][q] : acc[q][r];
            for (int r = 0; r < d; ++r)
                a.diag_raw[(int64_t)d * i + r] = out[r][r];
            for (int r = 0; r < d; ++r)
                for (int q = 0; q < d; ++q)
                    if (r != q && (ci[r] || ci[q]))
                        out[r][q] = 0.0;
        }
        else
        {
            double f[2][3][3], g[2][3][3];
            for (int L = 0; L < 2; ++L)
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q)
                    {
                        f[L][r][q] = 0.0;
                        g[L][r][q] = 0.0;
                    }
            for (int L = 0; L < 2; ++L)
            {
                const int aj = s.dir[L * kMaxConns + sl];
                const int olo = (L == 0) ? 0 : n0, ohi = (L == 0) ? n0 : nbi;
                // K_L(i, j): fdu2dxyz1/2(pi = i, pj = j)
                for (int o = olo; o < ohi; ++o)
                {
                    const double *co = s.o_cs + 3 * o;
                    const int hb = s.hop[o * kMaxConns + sl];
                    if (aj >= 0)
                    {
                        if (o == aj)
                        {
                            add_direct(f[L], d, s.o_D[o], s.o_Kn[o], s.o_Tv[o], co, s.o_S + 3 * o);
                            continue;
                        }
                        sub_other(f[L], d, s.o_D[aj], s.o_Tv[aj], s.o_cs + 3 * aj, s.o_D[o], s.o_Tv[o], co);
                    }
                    if (hb >= 0)
                    {
                        const int q = s.n_off[o] + hb;
                        sub_hop(f[L], d, s.o_D[o], s.o_Tv[o], co, s.n_D[q], s.n_Tv[q], s.n_cs + 3 * q);
                    }
                }
                // K_L(j, i): fdu2dxyz1/2(pi = j, pj = i), accumulated in j's orientation
                if (aj >= 0)
                {
                    const int jlo = s.n_off[aj], jhi = s.n_off[aj + 1];
                    const int rji = jlo + s.o_revpos[aj]; // bond j -> i
                    for (int q = jlo; q < jhi; ++q)
                    {
                        const double *cq = s.n_cs + 3 * q;
                        if (s.n_p2[q] == i)
                        {
                            add_direct(g[L], d, s.n_D[q], s.n_Kn[q], s.n_Tv[q], cq,
                                       a.cs_sum + 6 * (int64_t)i + 3 * L);
                            continue;
                        }
                        sub_other(g[L], d, s.n_D[rji], s.n_Tv[rji], s.n_cs + 3 * rji, s.n_D[q], s.n_Tv[q], cq);
                        const int xs = s.n_slot[q];
                        const int ax = (xs >= 0) ? s.dir[L * kMaxConns + xs] : -1;
                        if (ax >= 0)
                        {
                            const int rxi = s.n_off[ax] + s.o_revpos[ax]; // bond x -> i
                            sub_hop(g[L], d, s.n_D[q], s.n_Tv[q], cq, s.n_D[rxi], s.n_Tv[rxi], s.n_cs + 3 * rxi);
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
                        const int q = s.n_off[o] + hb;      // bond k -> j
                        const int bjk = s.n_rev[q];          // bond j -> k (global)
                        const int rki = s.n_off[o] + s.o_revpos[o]; // bond k -> i
                        const double cjk[3] = {a.cs[3 * (int64_t)bjk], a.cs[3 * (int64_t)bjk + 1],
                                               a.cs[3 * (int64_t)bjk + 2]};
                        sub_hop(g[L], d, a.bdamage[bjk], a.Tv[bjk], cjk, s.n_D[rki], s.n_Tv[rki], s.n_cs + 3 * rki);
                    }
                }
            }
            bool cj[3];
            const double dvj = a.damage_visual[j];
            for (int k = 0; k < 3; ++k)
                cj[k] = a.apply_bc && (k < d) && (a.cons[3 * j + k] == 1 || fabs(dvj - 1.0) < kEps);
            for (int r = 0; r < d; ++r)
                for (int q = 0; q < d; ++q)
                {
                    const double kij = f[0][r][q] + f[1][r][q];
                    const double kji = g[0][q][r] + g[1][q][r];
                    const double v = 0.5 * kij + 0.5 * kji;
                    out[r][q] = (ci[r] || cj[q]) ? 0.0 : v;
                }
        }
        double *dst = a.K + (sbase + sl) * d * d * kSlice + lane;
        for (int r = 0; r < d; ++r)
            for (int q = 0; q < d; ++q)
                dst[(r * d + q) * kSlice] = out[r][q];
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
                          double *__restrict__ K)
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
            K[(b * dim * dim + k * dim + k) * kSlice + pos % kSlice] = nd;
}

cudaError_t launch_assemble(Problem &p, bool apply_bc)
{
    AsmArgs a;
    a.n = p.n;
    a.dim = p.dim;
    a.mb = p.max_bonds;
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
    const size_t smem = asm_smem_bytes(a.mb);
    cudaError_t e = cudaFuncSetAttribute(k_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    k_assemble<<<p.n, kAsmThreads, smem, p.stream>>>(a);
    p.ctr.kernel_launches++;
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    if (apply_bc)
    {
        k_diag_norm<<<1, 1024, 0, p.stream>>>((int64_t)p.n * p.dim, p.diag_raw, p.scal);
        k_bc_diag<<<div_up(p.n, 256), 256, 0, p.stream>>>(p.n, p.dim, p.perm, p.slice_off, p.cstart, p.nlq, p.cons,
                                                          p.damage_visual, p.scal, p.K);
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
