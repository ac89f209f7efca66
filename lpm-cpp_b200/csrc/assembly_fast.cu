// Global stiffness assembly, fast form (the default; lpmgpu_set_assembly_exact selects the
// bit-exact kernel of assembly.cu).  Same matrix as the reference's
// Stiffness::calcStiffness2D/3D (include/stiffness.h:198-361) over localStiffnessANA
// (include/derivative.h:8-239), restated so that every sum runs over precomputed lists and no
// lane walks bond paths of its own:
//
// For a connection j of particle i (j != i) and layer L, with T_b = (1 - D_b) Tv_b, S_x = the
// layer's cosine sum of x (cs_sum) and U_x = sum_b T_b cs_b over x's bonds of the layer:
//   * j a layer-L neighbour through own bond a (i -> j) with opposite bond r (j -> i):
//       K(i,j) += (1-D_a) c_a (x) (-(2 Kn_a + Tv_a) c_a + Tv_a S_j) - 1/2 V (x) c_a,
//                 V = T_a S_i + U_i - 2 T_a c_a           (derivative.h:53-99 for layer 0)
//       K(j,i)^T from the same terms of bond r, seen from j (S_j, U_j, S_i, c_r);
//     the "other bond" sum over i's remaining bonds (derivative.h:91-99) is the closed form V.
//   * every 2-hop path i -> k -> j (own bond a to k, k's bond b to j, both of layer L):
//       K(i,j)   -= 1/2 (T_a + T_b) c_a (x) c_b           (derivative.h:105-113, 128-136)
//       K(j,i)^T -= 1/2 (T_r(b) + T_r(a)) c_r(a) (x) c_r(b)
//     with r(x) the opposite bond.  When no bond is broken in one direction only, c_r(x) = -c_x,
//     and the two halves of the stored block merge into -(Ts_a + Ts_b)/4 c_a (x) c_b, Ts = T + T_r.
// The stored block is 1/2 K(i,j) + 1/2 K(j,i)^T, the value the reference's two scatters leave
// (stiffness.h:232-276); the self block is fdu2dxyz (derivative.h:8-45).
//
// Layout of the work: one warp per particle row (in sliced-ELL order, so the 32 rows of a slice
// are written at about the same time and their interleaved entries merge in L2).  Lanes own
// connection slots; each lane sums its slot's 2-hop paths from the precomputed path list (built
// once per problem: per slot, the (own bond, partner bond) pairs in a fixed order), so every sum
// is deterministic and no atomics are used.  The own bonds' cosines and Ts are staged in shared
// memory.  This file is compiled with FMA contraction (the exact kernel is not): the result
// agrees with the reference within rounding (about 1e-15 of max|K|), not bit for bit.
#include "lpm_internal.cuh"

namespace lpm
{

constexpr int kAsmWarps = 8;
constexpr int kPathWarps = 8;

__device__ __forceinline__ double wsum_d(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int slot_of(const int *conns, int nc, int x)
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

// Per assembly: T_b, Ts_b = T_b + T_r(b) per bond, U per particle and layer, and whether a bond
// is broken in one direction only (then the 2-hop terms take the opposite bonds' own cosines).
__global__ void __launch_bounds__(256) k_asm_prep(int n, const int *__restrict__ bstart, const int *__restrict__ nb0,
                                                  const int *__restrict__ brev, const double *__restrict__ Tv,
                                                  const double *__restrict__ bdamage, const double *__restrict__ cs,
                                                  double *__restrict__ T, double *__restrict__ Ts,
                                                  double *__restrict__ U, int *__restrict__ asym)
{
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * (blockDim.x >> 5);
    bool odd = false;
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nw)
    {
        const int b0 = bstart[i], b1 = b0 + nb0[i], be = bstart[i + 1];
        for (int L = 0; L < 2; ++L)
        {
            const int lo = L == 0 ? b0 : b1, hi = L == 0 ? b1 : be;
            double u0 = 0, u1 = 0, u2 = 0;
            for (int b = lo + lane; b < hi; b += 32)
            {
                const double Db = bdamage[b];
                const double t = (1 - Db) * Tv[b];
                const int rb = brev[b];
                const double Dr = bdamage[rb];
                T[b] = t;
                Ts[b] = t + (1 - Dr) * Tv[rb];
                odd |= (fabs(Db - 1.0) < kEps) != (fabs(Dr - 1.0) < kEps);
                u0 += t * cs[3 * (int64_t)b];
                u1 += t * cs[3 * (int64_t)b + 1];
                u2 += t * cs[3 * (int64_t)b + 2];
            }
            u0 = wsum_d(u0);
            u1 = wsum_d(u1);
            u2 = wsum_d(u2);
            if (lane == 0)
            {
                U[6 * (int64_t)i + 3 * L] = u0;
                U[6 * (int64_t)i + 3 * L + 1] = u1;
                U[6 * (int64_t)i + 3 * L + 2] = u2;
            }
        }
    }
    if (__any_sync(0xffffffffu, odd) && lane == 0)
        atomicExch(asym, 1);
}

// The 2-hop path lists (once per problem).  One warp per particle row i, conns(i) staged; for
// each own bond o in order, the partner k's bonds of o's layer (k -> j, j != i) in order are the
// paths of slot(j).  COUNT: per-slot counts (<= 255, else *err) and the row total.  FILL: the
// paths at row_off[i] + start(slot) + running count, as (partner bond b, own bond index o).
template <bool FILL>
__global__ void __launch_bounds__(32 * kPathWarps) k_asm_paths(int n, int maxc, const int *__restrict__ bstart,
                                                               const int *__restrict__ nb0, const int *__restrict__ bp2,
                                                               const int *__restrict__ cstart,
                                                               const int *__restrict__ conns,
                                                               unsigned char *__restrict__ cnt,
                                                               int64_t *__restrict__ row_off, int *__restrict__ pb,
                                                               unsigned char *__restrict__ pa, int *__restrict__ err)
{
    extern __shared__ int psm[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *sc = psm + (size_t)w * 3 * maxc, *f = sc + maxc, *st = f + maxc;
    const int nw = gridDim.x * kPathWarps;
    for (int i = blockIdx.x * kPathWarps + w; i < n; i += nw)
    {
        const int b0 = bstart[i], n0 = nb0[i], nbi = bstart[i + 1] - b0;
        const int c0 = cstart[i], nc = cstart[i + 1] - c0;
        for (int s = lane; s < nc; s += 32)
        {
            sc[s] = conns[c0 + s];
            f[s] = 0;
        }
        if (FILL)
        {
            int run = 0;
            for (int base = 0; base < nc; base += 32)
            {
                const int s = base + lane;
                const int v = s < nc ? (int)cnt[c0 + s] : 0;
                int x = v;
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o)
                        x += y;
                }
                if (s < nc)
                    st[s] = run + x - v;
                run += __shfl_sync(0xffffffffu, x, 31);
            }
        }
        __syncwarp();
        const int64_t base = FILL ? row_off[i] : 0;
        int total = 0;
        for (int o = 0; o < nbi; ++o)
        {
            const int k = bp2[b0 + o];
            const bool l0 = o < n0;
            const int klo = l0 ? bstart[k] : bstart[k] + nb0[k];
            const int khi = l0 ? bstart[k] + nb0[k] : bstart[k + 1];
            for (int q = klo + lane; q < khi; q += 32)
            {
                const int j = bp2[q];
                if (j == i)
                    continue;
                const int s = slot_of(sc, nc, j);
                if (s < 0)
                {
                    atomicExch(err, 1);
                    continue;
                }
                if (FILL)
                {
                    const int64_t at = base + st[s] + f[s];
                    pb[at] = q;
                    pa[at] = (unsigned char)o;
                }
                f[s] += 1; // the partners j of one bond list are distinct: no two lanes share s
                total += 1;
            }
            __syncwarp();
        }
        if (!FILL)
        {
            for (int s = lane; s < nc; s += 32)
            {
                if (f[s] > 255)
                    atomicExch(err, 2);
                cnt[c0 + s] = (unsigned char)min(f[s], 255);
            }
            for (int o = 16; o > 0; o >>= 1)
                total += __shfl_xor_sync(0xffffffffu, total, o);
            if (lane == 0)
                row_off[i] = total;
        }
        __syncwarp();
    }
}

// exclusive scan of v[0 .. n) in place into out[0 .. n] (out[n] = total); one block
__global__ void __launch_bounds__(1024) k_scan_rows(int n, const int64_t *__restrict__ v, int64_t *__restrict__ out)
{
    __shared__ int64_t sh[1024];
    const int t = threadIdx.x;
    const int64_t chunk = ((int64_t)n + blockDim.x - 1) / blockDim.x;
    const int64_t lo = min((int64_t)n, t * chunk), hi = min((int64_t)n, lo + chunk);
    int64_t s = 0;
    for (int64_t k = lo; k < hi; ++k)
        s += v[k];
    sh[t] = s;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1)
    {
        const int64_t y = t >= o ? sh[t - o] : 0;
        __syncthreads();
        sh[t] += y;
        __syncthreads();
    }
    int64_t run = sh[t] - s;
    for (int64_t k = lo; k < hi; ++k)
    {
        const int64_t x = v[k];
        out[k] = run;
        run += x;
    }
    if (t == (int)blockDim.x - 1)
        out[n] = sh[t];
}

struct FastArgs
{
    int n, maxb, maxc, apply_bc;
    const int *__restrict__ bstart, *__restrict__ nb0, *__restrict__ bp2, *__restrict__ brev;
    const int *__restrict__ cstart, *__restrict__ conns, *__restrict__ nlq, *__restrict__ cons;
    const int *__restrict__ perm;
    const int64_t *__restrict__ slice_off;
    const double *__restrict__ cs, *__restrict__ Kn, *__restrict__ Tv, *__restrict__ bdamage;
    const double *__restrict__ cs_sum, *__restrict__ damage_visual;
    const double *__restrict__ T, *__restrict__ Ts, *__restrict__ U;
    const int *__restrict__ asym;
    const unsigned char *__restrict__ cnt, *__restrict__ pa;
    const int64_t *__restrict__ row_off;
    const int *__restrict__ pb;
    double *__restrict__ K, *__restrict__ diag_raw;
    float *__restrict__ K32; // written too when not null (mixed precision)
};

template <int D>
__global__ void __launch_bounds__(32 * kAsmWarps, D == 2 ? 4 : 3) k_assemble_fast(FastArgs a)
{
    extern __shared__ __align__(16) unsigned char fsm[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // per warp: ca[3*maxb], ta[maxb], tsa[maxb], cra[3*maxb], tra[maxb] | sc[maxc], dirb[maxc], pst[maxc + 1]
    const size_t wd = 9 * (size_t)a.maxb;
    double *ca = reinterpret_cast<double *>(fsm) + wd * w, *ta = ca + 3 * a.maxb, *tsa = ta + a.maxb,
           *cra = tsa + a.maxb, *tra = cra + 3 * a.maxb;
    int *sc = reinterpret_cast<int *>(reinterpret_cast<double *>(fsm) + wd * kAsmWarps) + (size_t)w * (3 * a.maxc + 1),
        *dirb = sc + a.maxc, *pst = dirb + a.maxc;
    const int pos = blockIdx.x * kAsmWarps + w;
    if (pos >= a.n)
        return;
    const int i = a.perm[pos];
    const int row_lane = pos % kSlice;
    const int64_t sbase = a.slice_off[pos / kSlice];
    const int b0 = a.bstart[i], n0 = a.nb0[i], nbi = a.bstart[i + 1] - b0;
    const int c0 = a.cstart[i], nc = a.cstart[i + 1] - c0;
    const bool asym = *a.asym != 0;
    for (int s = lane; s < nc; s += 32)
    {
        sc[s] = a.conns[c0 + s];
        dirb[s] = -1;
    }
    for (int o = lane; o < nbi; o += 32)
    {
        const int b = b0 + o;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            ca[3 * o + c] = a.cs[3 * (int64_t)b + c];
        ta[o] = a.T[b];
        tsa[o] = a.Ts[b];
        if (asym)
        {
            const int rb = a.brev[b];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                cra[3 * o + c] = a.cs[3 * (int64_t)rb + c];
            tra[o] = a.T[rb];
        }
    }
    // per-slot path starts: exclusive scan of the counts
    {
        int run = 0;
        for (int base = 0; base < nc; base += 32)
        {
            const int s = base + lane;
            const int v = s < nc ? (int)a.cnt[c0 + s] : 0;
            int x = v;
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o)
                    x += y;
            }
            if (s < nc)
                pst[s] = run + x - v;
            run += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0)
            pst[nc] = run;
    }
    __syncwarp();
    for (int o = lane; o < nbi; o += 32)
    {
        const int s = slot_of(sc, nc, a.bp2[b0 + o]);
        if (s >= 0)
            dirb[s] = o;
    }
    // the layer's cosine sum S and U of particle i (read through L1 where a layer is chosen at run time)
    const double *Si_g = a.cs_sum + 6 * (int64_t)i, *Ui_g = a.U + 6 * (int64_t)i;
    // self block (fdu2dxyz, derivative.h:8-45): sum over the own bonds of
    // (1-D) [(2 Kn + Tv) c_r c_q + Tv c_r S[q]] for r <= q, mirrored
    double self[D][D];
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
        for (int q = 0; q < D; ++q)
            self[r][q] = 0.0;
    for (int o = lane; o < nbi; o += 32)
    {
        const int b = b0 + o;
        const int L = o < n0 ? 0 : 1;
        const double Dm = a.bdamage[b], Kn = a.Kn[b], Tv = a.Tv[b];
        const double *c = ca + 3 * o;
        const double f = (1 - Dm) * (2 * Kn + Tv), g = (1 - Dm) * Tv;
        double S[D];
#pragma unroll
        for (int q = 0; q < D; ++q)
            S[q] = Si_g[3 * L + q];
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int q = 0; q < D; ++q)
                if (r <= q)
                    self[r][q] += f * c[r] * c[q] + g * c[r] * S[q];
    }
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
        for (int q = 0; q < D; ++q)
            if (r <= q)
                self[r][q] = wsum_d(self[r][q]);
    __syncwarp();
    const int selfslot = nc - a.nlq[i];
    const double dvi = a.damage_visual[i];
    bool ci[D];
#pragma unroll
    for (int k = 0; k < D; ++k)
        ci[k] = a.apply_bc && (a.cons[3 * i + k] == 1 || fabs(dvi - 1.0) < kEps);
    const int64_t rbase = a.row_off[i];

    for (int s = lane; s < nc; s += 32)
    {
        const int j = sc[s];
        double acc[D][D];
        if (s == selfslot)
        {
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int q = 0; q < D; ++q)
                    acc[r][q] = r <= q ? self[r][q] : self[q][r];
#pragma unroll
            for (int r = 0; r < D; ++r)
            {
                a.diag_raw[(int64_t)D * i + r] = acc[r][r];
#pragma unroll
                for (int q = 0; q < D; ++q)
                    if (r != q && (ci[r] || ci[q]))
                        acc[r][q] = 0.0;
            }
        }
        else
        {
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int q = 0; q < D; ++q)
                    acc[r][q] = 0.0;
            const int o = dirb[s];
            if (o >= 0)
            {
                // own bond a = i -> j and its opposite r = j -> i
                const int b = b0 + o, L = o < n0 ? 0 : 1, rb = a.brev[b];
                const double *c = ca + 3 * o;
                const double Da = a.bdamage[b], Kna = a.Kn[b], Tva = a.Tv[b], Taa = ta[o];
                const double Dr = a.bdamage[rb], Knr = a.Kn[rb], Tvr = a.Tv[rb], Trr = a.T[rb];
                double cr[3], Sj[3], Si[3], V[3], W[3];
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    cr[k] = a.cs[3 * (int64_t)rb + k];
                    Sj[k] = a.cs_sum[6 * (int64_t)j + 3 * L + k];
                    Si[k] = Si_g[3 * L + k];
                    V[k] = Taa * Si[k] + Ui_g[3 * L + k] - 2 * Taa * c[k];
                    W[k] = Trr * Sj[k] + a.U[6 * (int64_t)j + 3 * L + k] - 2 * Trr * cr[k];
                }
                const double fa = 2 * Kna + Tva, fr = 2 * Knr + Tvr;
#pragma unroll
                for (int r = 0; r < D; ++r)
#pragma unroll
                    for (int q = 0; q < D; ++q)
                    {
                        const double kij = (1 - Da) * c[r] * (Tva * Sj[q] - fa * c[q]) - 0.5 * V[r] * c[q];
                        const double kji = (1 - Dr) * cr[q] * (Tvr * Si[r] - fr * cr[r]) - 0.5 * W[q] * cr[r];
                        acc[r][q] += 0.5 * kij + 0.5 * kji;
                    }
            }
            const int p0 = pst[s], p1 = pst[s + 1];
            for (int p = p0; p < p1; ++p)
            {
                const int q = a.pb[rbase + p];
                const int oa = a.pa[rbase + p];
                const double *cA = ca + 3 * oa;
                double cB[3];
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    cB[k] = a.cs[3 * (int64_t)q + k];
                if (!asym)
                {
                    const double wgt = -0.25 * (tsa[oa] + a.Ts[q]);
#pragma unroll
                    for (int r = 0; r < D; ++r)
#pragma unroll
                        for (int c2 = 0; c2 < D; ++c2)
                            acc[r][c2] += wgt * cA[r] * cB[c2];
                }
                else
                {
                    const int rq = a.brev[q];
                    const double *cRA = cra + 3 * oa;
                    double cRB[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        cRB[k] = a.cs[3 * (int64_t)rq + k];
                    const double w1 = -0.25 * (ta[oa] + a.T[q]), w2 = -0.25 * (tra[oa] + a.T[rq]);
#pragma unroll
                    for (int r = 0; r < D; ++r)
#pragma unroll
                        for (int c2 = 0; c2 < D; ++c2)
                            acc[r][c2] += w1 * cA[r] * cB[c2] + w2 * cRA[r] * cRB[c2];
                }
            }
            const double dvj = a.damage_visual[j];
#pragma unroll
            for (int q = 0; q < D; ++q)
            {
                const bool cj = a.apply_bc && (a.cons[3 * j + q] == 1 || fabs(dvj - 1.0) < kEps);
#pragma unroll
                for (int r = 0; r < D; ++r)
                    if (ci[r] || cj)
                        acc[r][q] = 0.0;
            }
        }
        const int64_t e0 = (sbase + s) * D * D * kSlice + row_lane;
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int q = 0; q < D; ++q)
            {
                a.K[e0 + (r * D + q) * kSlice] = acc[r][q];
                if (a.K32)
                    a.K32[e0 + (r * D + q) * kSlice] = (float)acc[r][q];
            }
    }
}

static size_t fast_smem(const Problem &p)
{
    return sizeof(double) * 9 * (size_t)p.max_bonds * kAsmWarps +
           sizeof(int) * (3 * (size_t)p.max_conns + 1) * kAsmWarps;
}

// Builds the 2-hop path lists (once per problem).  On success p.asm_fast is set; when a slot
// has more than 255 paths the problem keeps the exact kernel.
cudaError_t setup_fast_assembly(Problem &p)
{
    p.asm_fast = false;
    if (p.max_bonds > 255 || p.max_bonds < 1)
        return cudaSuccess;
    cudaError_t e;
    if ((e = dalloc(p, &p.asm_T, (size_t)p.nbonds)) != cudaSuccess)
        return e;
    if ((e = dalloc(p, &p.asm_Ts, (size_t)p.nbonds)) != cudaSuccess)
        return e;
    if ((e = dalloc(p, &p.asm_U, 6 * (size_t)p.n)) != cudaSuccess)
        return e;
    if ((e = dalloc(p, &p.asm_cnt, (size_t)p.nnzb)) != cudaSuccess)
        return e;
    if ((e = dalloc(p, &p.asm_row, (size_t)p.n + 1)) != cudaSuccess)
        return e;
    int64_t *counts = nullptr;
    int *err = nullptr;
    if ((e = dalloc(p, &counts, (size_t)p.n)) != cudaSuccess)
        return e;
    if ((e = dalloc(p, &err, 1)) != cudaSuccess)
        return e;
    const size_t psmem = sizeof(int) * 3 * (size_t)p.max_conns * kPathWarps;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(div_up(p.n, kPathWarps), (int64_t)p.num_sms * 16));
    k_asm_paths<false><<<grid, 32 * kPathWarps, psmem, p.stream>>>(p.n, p.max_conns, p.bstart, p.nb0, p.bp2,
                                                                   p.cstart, p.conns, p.asm_cnt, counts, nullptr,
                                                                   nullptr, err);
    k_scan_rows<<<1, 1024, 0, p.stream>>>(p.n, counts, p.asm_row);
    int64_t total = 0;
    int herr = 0;
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(&total, p.asm_row + p.n, sizeof(int64_t), cudaMemcpyDeviceToHost, p.stream)) !=
        cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, p.stream)) != cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(p.stream)) != cudaSuccess)
        return e;
    if (herr != 0)
        return cudaSuccess; // a slot with more than 255 paths: the exact kernel stays in use
    if ((e = dalloc(p, &p.asm_pb, (size_t)std::max<int64_t>(total, 1))) != cudaSuccess)
        return e;
    if ((e = dalloc(p, &p.asm_pa, (size_t)std::max<int64_t>(total, 1))) != cudaSuccess)
        return e;
    k_asm_paths<true><<<grid, 32 * kPathWarps, psmem, p.stream>>>(p.n, p.max_conns, p.bstart, p.nb0, p.bp2, p.cstart,
                                                                  p.conns, p.asm_cnt, p.asm_row, p.asm_pb, p.asm_pa,
                                                                  err);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, p.stream)) != cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(p.stream)) != cudaSuccess)
        return e;
    p.asm_paths = total;
    p.asm_asym = err; // reused as the per-assembly "broken in one direction" flag
    p.asm_fast = herr == 0;
    return cudaSuccess;
}

cudaError_t launch_assemble_fast(Problem &p, bool apply_bc, bool write_k32)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(p.asm_asym, 0, sizeof(int), p.stream)) != cudaSuccess)
        return e;
    const int pgrid = (int)std::max<int64_t>(1, std::min<int64_t>(div_up(p.n, 8), (int64_t)p.num_sms * 16));
    k_asm_prep<<<pgrid, 256, 0, p.stream>>>(p.n, p.bstart, p.nb0, p.brev, p.Tv, p.bdamage, p.cs, p.asm_T, p.asm_Ts,
                                            p.asm_U, p.asm_asym);
    FastArgs a;
    a.n = p.n;
    a.maxb = p.max_bonds;
    a.maxc = p.max_conns;
    a.apply_bc = apply_bc ? 1 : 0;
    a.bstart = p.bstart;
    a.nb0 = p.nb0;
    a.bp2 = p.bp2;
    a.brev = p.brev;
    a.cstart = p.cstart;
    a.conns = p.conns;
    a.nlq = p.nlq;
    a.cons = p.cons;
    a.perm = p.perm;
    a.slice_off = p.slice_off;
    a.cs = p.cs;
    a.Kn = p.Kn;
    a.Tv = p.Tv;
    a.bdamage = p.bdamage;
    a.cs_sum = p.cs_sum;
    a.damage_visual = p.damage_visual;
    a.T = p.asm_T;
    a.Ts = p.asm_Ts;
    a.U = p.asm_U;
    a.asym = p.asm_asym;
    a.cnt = p.asm_cnt;
    a.pa = p.asm_pa;
    a.row_off = p.asm_row;
    a.pb = p.asm_pb;
    a.K = p.K;
    a.diag_raw = p.diag_raw;
    a.K32 = write_k32 ? p.K32 : nullptr;
    const size_t smem = fast_smem(p);
    const int grid = div_up(p.n, kAsmWarps);
    if (p.dim == 2)
    {
        if ((e = cudaFuncSetAttribute(k_assemble_fast<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
            return e;
        k_assemble_fast<2><<<grid, 32 * kAsmWarps, smem, p.stream>>>(a);
    }
    else
    {
        if ((e = cudaFuncSetAttribute(k_assemble_fast<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
            return e;
        k_assemble_fast<3><<<grid, 32 * kAsmWarps, smem, p.stream>>>(a);
    }
    p.ctr.kernel_launches += 2;
    return cudaGetLastError();
}

} // namespace lpm
