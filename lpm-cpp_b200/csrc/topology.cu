// Device construction of the particle topology: bonds, opposite-bond index, connection
// lists, the sliced-ELL row order and column slots of the solver's stiffness, and the 1-based
// upper-CSR pointers of the reference.  Restates, on the device:
//   Bond(p1,p2,layer,dis)          include/bond.h:59-72
//   Assembly::createBonds          include/assembly.h:213-234  (O(N^2) in the reference;
//                                  here a radix-sorted cell grid, same lists, same order)
//   Assembly::updateConnections    include/assembly.h:237-266
//   Stiffness::initialize          include/stiffness.h:55-71   (K_pointer)
// The distance is sqrt(dx*dx + dy*dy + dz*dz) evaluated in that order (particle.h:277-280,
// where the compiler folds pow(x, 2) into x*x), so the bond/layer decisions are identical.

#include <algorithm>
#include <climits>
#include <cmath>
#include <map>
#include <vector>

#include "lpm_internal.cuh"

namespace lpm
{

Cell make_cell(int lattice, double r)
{
    Cell c;
    c.lattice = lattice;
    c.radius = r;
    const double s2 = std::sqrt(2.0), s3 = std::sqrt(3.0);
    switch (lattice)
    {
    case LPMGPU_SQUARE2D:
    {
        const double e[9] = {1. / 2., -1. / 2., 0., 0., 0., 1. / 2., 0., 1. / 12., -1. / 12.};
        std::copy(e, e + 9, c.el);
        c.dim = 2;
        c.nneighbors = 8;
        c.cutoff[0] = 2.0 * r;
        c.cutoff[1] = 2.0 * s2 * r;
        c.pvol = 4 * (r * r);
        break;
    }
    case LPMGPU_HEXAGON2D:
    {
        const double e[9] = {s3 / 12.0, -s3 / 12.0, 0., -s3 / 144.0, s3 / 48.0, 0.0, 0.0, 0.0, 1.0};
        std::copy(e, e + 9, c.el);
        c.dim = 2;
        c.nneighbors = 12;
        c.cutoff[0] = 2.0 * r;
        c.cutoff[1] = 2.0 * s3 * r;
        c.pvol = 2 * s3 * (r * r);
        break;
    }
    case LPMGPU_SC3D:
    {
        const double e[9] = {1, -1, -1.0, 0.0, 0.0, 1., 0.0, 1 / 18.0, -1 / 18.0};
        std::copy(e, e + 9, c.el);
        c.dim = 3;
        c.nneighbors = 18;
        c.cutoff[0] = 2.0 * r;
        c.cutoff[1] = 2.0 * s2 * r;
        c.pvol = std::pow(2 * r, 3);
        break;
    }
    case LPMGPU_FCC3D:
    {
        const double e[9] = {0.0, 0.0, s2, s2 / 4, -s2 / 4, -s2 / 4, 0.0, s2 / 24, -s2 / 24};
        std::copy(e, e + 9, c.el);
        c.dim = 3;
        c.nneighbors = 18;
        c.cutoff[0] = 2.0 * r;
        c.cutoff[1] = 2.0 * s2 * r;
        c.pvol = 4.0 * s2 * std::pow(r, 3);
        break;
    }
    default:
    {
        const double e[9] = {0.0, 0.0, s3, 1 / s3, -1 / s3, 0., 0.0, s3 / 14, s3 / 14};
        std::copy(e, e + 9, c.el);
        c.dim = 3;
        c.nneighbors = 14;
        c.cutoff[0] = 2.0 * r;
        c.cutoff[1] = 4.0 / s3 * r;
        c.pvol = 32.0 * s3 / 9.0 * std::pow(r, 3);
        break;
    }
    }
    return c;
}

// Ce of plane stress / strain, then KnTv = alpha * (el_mapping . Ce) with the in-order
// dot product and alpha = 1 (2D) or radius (3D): particle_elastic.h:76-90
void kntv(const Cell &c, int plane_stress, double E, double mu, double out[3])
{
    double Ce[3];
    if (!plane_stress)
    {
        Ce[0] = E * (1.0 - mu) / (1.0 + mu) / (1.0 - 2.0 * mu);
        Ce[1] = E * mu / (1.0 + mu) / (1.0 - 2.0 * mu);
        Ce[2] = E / 2.0 / (1.0 + mu);
    }
    else
    {
        Ce[0] = E / (1.0 - mu) / (1.0 + mu);
        Ce[1] = E * mu / (1.0 + mu) / (1.0 - mu);
        Ce[2] = E / 2.0 / (1.0 + mu);
    }
    const double alpha = (c.dim == 2) ? 1.0 : c.radius;
    for (int r = 0; r < 3; ++r)
    {
        double s = 0.0;
        for (int k = 0; k < 3; ++k)
            s += c.el[3 * r + k] * Ce[k];
        out[r] = alpha * s;
    }
}

// setParticleProperty's (C11, C12, C44) overload (particle_elastic.h:110-140): the same mapping
// from given elastic constants
void kntv_cij(const Cell &c, const double Ce[3], double out[3])
{
    const double alpha = (c.dim == 2) ? 1.0 : c.radius;
    for (int r = 0; r < 3; ++r)
    {
        double s = 0.0;
        for (int k = 0; k < 3; ++k)
            s += c.el[3 * r + k] * Ce[k];
        out[r] = alpha * s;
    }
}

__device__ __forceinline__ double pdist(const double *a, const double *b)
{
    const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

struct Grid
{
    double lo[3];
    double h;
    int nc[3];
};

__device__ __forceinline__ int cell_coord(double v, double lo, double h, int nc)
{
    int c = (int)floor((v - lo) / h);
    return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_cell_keys(int n, const double *__restrict__ xyz, Grid g, int *__restrict__ key,
                            int *__restrict__ ids)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int cx = cell_coord(xyz[3 * i], g.lo[0], g.h, g.nc[0]);
    int cy = cell_coord(xyz[3 * i + 1], g.lo[1], g.h, g.nc[1]);
    int cz = cell_coord(xyz[3 * i + 2], g.lo[2], g.h, g.nc[2]);
    key[i] = (cz * g.nc[1] + cy) * g.nc[0] + cx;
    ids[i] = i;
}

__global__ void k_cell_bounds(int n, const int *__restrict__ skey, int *__restrict__ cbeg, int *__restrict__ cend)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n)
        return;
    int k = skey[q];
    if (q == 0 || skey[q - 1] != k)
        cbeg[k] = q;
    if (q == n - 1 || skey[q + 1] != k)
        cend[k] = q + 1;
}

// Assembly::createBonds: candidates with d < 1.01*cutoff1, i != j; layer 0 when
// d < 1.01*cutoff0.  Output padded [n][kMaxBonds], layer-0 ids then layer-1 ids, ascending.
__global__ void k_bonds_find(int n, const double *__restrict__ xyz, Grid g, const int *__restrict__ sid,
                             const int *__restrict__ cbeg, const int *__restrict__ cend, double rc0, double rc1,
                             int *__restrict__ pad_id, double *__restrict__ pad_d, int *__restrict__ nb,
                             int *__restrict__ nb0, Scalars *scal)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int cid[kMaxBonds];
    double cd[kMaxBonds];
    unsigned lay = 0; // bit q = layer of candidate q
    int m = 0;
    const double xi[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    int cx = cell_coord(xi[0], g.lo[0], g.h, g.nc[0]);
    int cy = cell_coord(xi[1], g.lo[1], g.h, g.nc[1]);
    int cz = cell_coord(xi[2], g.lo[2], g.h, g.nc[2]);
    bool overflow = false;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
            {
                int x = cx + dx, y = cy + dy, z = cz + dz;
                if (x < 0 || y < 0 || z < 0 || x >= g.nc[0] || y >= g.nc[1] || z >= g.nc[2])
                    continue;
                int c = (z * g.nc[1] + y) * g.nc[0] + x;
                for (int q = cbeg[c]; q < cend[c]; ++q)
                {
                    int j = sid[q];
                    const double xj[3] = {xyz[3 * j], xyz[3 * j + 1], xyz[3 * j + 2]};
                    double d = pdist(xi, xj);
                    if ((d < rc1) && (i != j))
                    {
                        if (m == kMaxBonds)
                        {
                            overflow = true;
                            continue;
                        }
                        // insertion by id keeps the list ascending
                        int pos = m;
                        while (pos > 0 && cid[pos - 1] > j)
                        {
                            cid[pos] = cid[pos - 1];
                            cd[pos] = cd[pos - 1];
                            pos--;
                        }
                        cid[pos] = j;
                        cd[pos] = d;
                        m++;
                    }
                }
            }
    if (overflow)
        atomicExch(&scal->err, 1);
    for (int q = 0; q < m; ++q)
        if (!(cd[q] < rc0))
            lay |= 1u << q;
    int w = 0, c0 = 0;
    for (int L = 0; L < 2; ++L)
        for (int q = 0; q < m; ++q)
            if (((lay >> q) & 1u) == (unsigned)L)
            {
                pad_id[(int64_t)i * kMaxBonds + w] = cid[q];
                pad_d[(int64_t)i * kMaxBonds + w] = cd[q];
                w++;
                c0 += (L == 0);
            }
    nb[i] = m;
    nb0[i] = c0;
}

// distances of caller-supplied bonds (Assembly::readBond computes them the same way, assembly.h:416)
__global__ void k_bonds_dist(int n, const double *__restrict__ xyz, const int *__restrict__ pad_id,
                             const int *__restrict__ nb, double *__restrict__ pad_d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    for (int q = 0; q < nb[i]; ++q)
    {
        const int j = pad_id[(int64_t)i * kMaxBonds + q];
        pad_d[(int64_t)i * kMaxBonds + q] = pdist(xyz + 3 * i, xyz + 3 * j);
    }
}

// Bond(p1,p2,layer,dis) (bond.h:59-72) and setParticleProperty's Kn/Tv assignment
// (particle_elastic.h:92-107): hexagonal lattices use Kn = KnTv[0], Tv = KnTv[1] for both layers
__global__ void k_bonds_fill(int n, const double *__restrict__ xyz, const int *__restrict__ pad_id,
                             const double *__restrict__ pad_d, const int *__restrict__ nb,
                             const int *__restrict__ nb0, const int *__restrict__ bstart, int hex, double k0,
                             double k1, double k2, int *__restrict__ bp2, double *__restrict__ dis0,
                             double *__restrict__ dis, double *__restrict__ dis_last, double *__restrict__ cs,
                             double *__restrict__ Kn, double *__restrict__ Tv)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int b0 = bstart[i];
    for (int q = 0; q < nb[i]; ++q)
    {
        const int b = b0 + q, j = pad_id[(int64_t)i * kMaxBonds + q];
        const double d = pad_d[(int64_t)i * kMaxBonds + q];
        const int layer = (q < nb0[i]) ? 0 : 1;
        bp2[b] = j;
        dis0[b] = d;
        dis[b] = d;
        dis_last[b] = d;
        for (int k = 0; k < 3; ++k)
            cs[3 * (int64_t)b + k] = (xyz[3 * i + k] - xyz[3 * j + k]) / d;
        if (hex)
        {
            Kn[b] = k0;
            Tv[b] = k1;
        }
        else
        {
            Kn[b] = layer == 0 ? k0 : k1;
            Tv[b] = k2;
        }
    }
}

// opposite bond: the first bond in p2's same-layer list that points back (particle.h:207-209)
__global__ void k_bonds_rev(int n, const int *__restrict__ bstart, const int *__restrict__ nb0,
                            const int *__restrict__ bp2, int *__restrict__ brev, Scalars *scal)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int b0 = bstart[i], b1 = b0 + nb0[i], be = bstart[i + 1];
    for (int b = b0; b < be; ++b)
    {
        const int j = bp2[b];
        const int L = (b < b1) ? 0 : 1;
        const int lo = (L == 0) ? bstart[j] : bstart[j] + nb0[j];
        const int hi = (L == 0) ? bstart[j] + nb0[j] : bstart[j + 1];
        int r = -1;
        for (int c = lo; c < hi; ++c)
            if (bp2[c] == i)
            {
                r = c;
                break;
            }
        brev[b] = r;
        if (r < 0)
            atomicExch(&scal->err, 2);
    }
}

// Assembly::updateConnections: conns(i) = sorted unique union over layers of N_L(i) and
// N_L(N_L(i)); nconn_largeq = #{j in conns(i), j >= i}.  One warp per particle: gather the
// candidates into shared memory, bitonic sort, compact the distinct ids.
__global__ void k_conns(int n, const int *__restrict__ bstart, const int *__restrict__ nb0,
                        const int *__restrict__ bp2, int *__restrict__ pad_c, int *__restrict__ nconn,
                        int *__restrict__ nlq, Scalars *scal)
{
    extern __shared__ int s_cand[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int i = blockIdx.x * (blockDim.x >> 5) + wib;
    if (i >= n)
        return;
    int *a = s_cand + wib * kMaxCand;
    const int b0 = bstart[i], nbi = bstart[i + 1] - b0, n0 = nb0[i];
    // lane q handles own bond q (nbi <= kMaxBonds == 32)
    int k = -1, L = 0, lo = 0, cnt = 0;
    if (lane < nbi)
    {
        k = bp2[b0 + lane];
        L = (lane < n0) ? 0 : 1;
        lo = (L == 0) ? bstart[k] : bstart[k] + nb0[k];
        const int hi = (L == 0) ? bstart[k] + nb0[k] : bstart[k + 1];
        cnt = 1 + (hi - lo);
    }
    int off = cnt;
    for (int d = 1; d < 32; d <<= 1)
    {
        int v = __shfl_up_sync(0xffffffffu, off, d);
        if (lane >= d)
            off += v;
    }
    const int total = __shfl_sync(0xffffffffu, off, 31);
    off -= cnt;
    if (total > kMaxCand)
    {
        if (lane == 0)
            atomicExch(&scal->err, 3);
        return;
    }
    if (lane < nbi)
    {
        a[off] = k;
        for (int c = 0; c < cnt - 1; ++c)
            a[off + 1 + c] = bp2[lo + c];
    }
    int m = 32;
    while (m < total)
        m <<= 1;
    for (int q = total + lane; q < m; q += 32)
        a[q] = INT_MAX;
    __syncwarp();
    for (int kk = 2; kk <= m; kk <<= 1)
        for (int j = kk >> 1; j > 0; j >>= 1)
        {
            for (int q = lane; q < m; q += 32)
            {
                int r = q ^ j;
                if (r > q)
                {
                    int x = a[q], y = a[r];
                    bool up = (q & kk) == 0;
                    if ((x > y) == up)
                    {
                        a[q] = y;
                        a[r] = x;
                    }
                }
            }
            __syncwarp();
        }
    int base = 0, ge = 0;
    for (int q0 = 0; q0 < m; q0 += 32)
    {
        const int q = q0 + lane;
        const int v = a[q];
        const bool keep = (v != INT_MAX) && (q == 0 || a[q - 1] != v);
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        const int pos = base + __popc(bal & ((1u << lane) - 1u));
        if (keep && pos < kMaxConns)
            pad_c[(int64_t)i * kMaxConns + pos] = v;
        base += __popc(bal);
        ge += __popc(__ballot_sync(0xffffffffu, keep && v >= i));
    }
    if (lane == 0)
    {
        if (base > kMaxConns || nbi == 0)
            atomicExch(&scal->err, 4);
        nconn[i] = base;
        nlq[i] = ge;
    }
}

// per particle: sum over its bonds of the partner's same-layer bond count (assembly staging size)
__global__ void k_records(int n, const int *__restrict__ bstart, const int *__restrict__ nb0,
                          const int *__restrict__ bp2, int *__restrict__ nrec)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int t = 0;
    for (int b = bstart[i]; b < bstart[i + 1]; ++b)
    {
        const int k = bp2[b];
        t += (b < bstart[i] + nb0[i]) ? nb0[k] : (bstart[k + 1] - bstart[k] - nb0[k]);
    }
    nrec[i] = t;
}

__global__ void k_conns_fill(int n, const int *__restrict__ pad_c, const int *__restrict__ cstart,
                             int *__restrict__ conns)
{
    int i = blockIdx.x;
    if (i >= n)
        return;
    const int c0 = cstart[i], m = cstart[i + 1] - c0;
    for (int q = threadIdx.x; q < m; q += blockDim.x)
        conns[c0 + q] = pad_c[(int64_t)i * kMaxConns + q];
}

// K_pointer[i+1] - K_pointer[i] = dim^2 * nconn_largeq - (dim == 2 ? 1 : 3)  (stiffness.h:59-65)
__global__ void k_kp_counts(int n, int dim, const int *__restrict__ nlq, int64_t *__restrict__ v)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        v[i] = (int64_t)dim * dim * nlq[i] - (dim == 2 ? 1 : 3);
    if (i == n)
        v[i] = 0;
}

// ---- sliced-ELL row order and column slots
__global__ void k_sell_keys(int n, const int *__restrict__ cstart, int *__restrict__ key, int *__restrict__ ids)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    key[i] = kMaxConns - (cstart[i + 1] - cstart[i]);
    ids[i] = i;
}

__global__ void k_sell_width(int n, int nslices, const int *__restrict__ perm, const int *__restrict__ cstart,
                             const int *__restrict__ iperm_unused, int64_t *__restrict__ width)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nslices)
    {
        const int i = perm[s * kSlice]; // a slice's rows are in descending count order
        width[s] = cstart[i + 1] - cstart[i];
    }
    if (s == nslices)
        width[s] = 0;
}

// perm_out's slice s' holds the 32 rows of perm's slice order[s'] (whole slices move)
__global__ void k_sell_move(int nmove, const int *__restrict__ order, const int *__restrict__ perm,
                            int *__restrict__ perm_out)
{
    const int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= (int64_t)nmove * kSlice)
        return;
    const int s = (int)(pos / kSlice), lane = (int)(pos % kSlice);
    perm_out[pos] = perm[(int64_t)order[s] * kSlice + lane];
}

__global__ void k_sell_fill(int n, int nslices, const int *__restrict__ perm, const int *__restrict__ cstart,
                            const int *__restrict__ conns, const int64_t *__restrict__ off, int *__restrict__ iperm,
                            int *__restrict__ col_sell)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= nslices * kSlice)
        return;
    const int s = pos / kSlice, lane = pos % kSlice;
    const int64_t o = off[s];
    const int w = (int)(off[s + 1] - o);
    if (pos >= n)
    {
        for (int k = 0; k < w; ++k)
            col_sell[(o + k) * kSlice + lane] = 0;
        return;
    }
    const int i = perm[pos];
    iperm[i] = pos;
    const int c0 = cstart[i], m = cstart[i + 1] - c0;
    for (int k = 0; k < w; ++k)
        col_sell[(o + k) * kSlice + lane] = (k < m) ? conns[c0 + k] : i;
}

// Spreads each slice width over the slice order.  The row sort puts the short rows of boundary
// particles last, so a problem's narrow slices, whose rows are scattered over the lattice and
// cost more per block slot (uncoalesced vector accesses), would all fall to the last blocks of
// any split of its slices by block slots.  Whole slices are reordered (rows within a slice, and
// so every row's columns and values, stay as they are): slice s of width class c and rank r in
// that class gets key (r + 1/2) / |c|, and slices are ordered by key (then width descending, then
// old position), which places each class evenly along the order.  A partial last slice stays
// last (its idle lanes are the positions >= n).  Applied to 2D lattices: on the 64 notched plates
// it took the batched CG from 4.90 s to 4.00 s, while on the 3D headline cube the single-problem
// CG, whose blocks take contiguous slice ranges that share neighbours in L1, lost 3.5% with it.
static cudaError_t spread_slices(Problem &p, int64_t *width)
{
    const int nmove = (p.n % kSlice == 0) ? p.nslices : p.nslices - 1;
    if (nmove < 2)
        return cudaSuccess;
    std::vector<int64_t> w(nmove);
    cudaError_t e = cudaMemcpyAsync(w.data(), width, sizeof(int64_t) * nmove, cudaMemcpyDeviceToHost, p.stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(p.stream);
    if (e != cudaSuccess)
        return e;
    std::map<int64_t, int> count, seen;
    for (int64_t x : w)
        count[x]++;
    std::vector<std::pair<double, int>> key(nmove);
    for (int s = 0; s < nmove; ++s)
        key[s] = {(seen[w[s]]++ + 0.5) / count[w[s]], s};
    std::stable_sort(key.begin(), key.end(), [&](const std::pair<double, int> &a, const std::pair<double, int> &b) {
        if (a.first != b.first)
            return a.first < b.first;
        if (w[a.second] != w[b.second])
            return w[a.second] > w[b.second];
        return a.second < b.second;
    });
    std::vector<int> order(nmove);
    std::vector<int64_t> wnew(nmove);
    bool moved = false;
    for (int s = 0; s < nmove; ++s)
    {
        order[s] = key[s].second;
        wnew[s] = w[order[s]];
        moved = moved || order[s] != s;
    }
    if (!moved)
        return cudaSuccess;
    int *d_order = nullptr, *perm2 = nullptr;
    if ((e = cudaMallocAsync(&d_order, sizeof(int) * nmove, p.stream)) != cudaSuccess)
        return e;
    if ((e = cudaMallocAsync(&perm2, sizeof(int) * (size_t)nmove * kSlice, p.stream)) != cudaSuccess)
        return e;
    e = cudaMemcpyAsync(d_order, order.data(), sizeof(int) * nmove, cudaMemcpyHostToDevice, p.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(width, wnew.data(), sizeof(int64_t) * nmove, cudaMemcpyHostToDevice, p.stream);
    if (e == cudaSuccess)
    {
        const int T = 256;
        k_sell_move<<<div_up((int64_t)nmove * kSlice, T), T, 0, p.stream>>>(nmove, d_order, p.perm, perm2);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p.perm, perm2, sizeof(int) * (size_t)nmove * kSlice, cudaMemcpyDeviceToDevice, p.stream);
    // the host vectors feed asynchronous copies: wait for them before they go out of scope
    const cudaError_t e2 = cudaStreamSynchronize(p.stream);
    cudaFreeAsync(d_order, p.stream);
    cudaFreeAsync(perm2, p.stream);
    return e != cudaSuccess ? e : e2;
}

template <typename T>
static cudaError_t exclusive_scan(Problem &p, const T *in, T *out, int count)
{
    return prim_exclusive_scan(p.stream, in, out, count);
}

static cudaError_t reduce_max(Problem &p, const int *in, int count, int *host_out)
{
    int *dmax = nullptr;
    cudaError_t e = cudaMallocAsync(&dmax, sizeof(int), p.stream);
    if (e != cudaSuccess)
        return e;
    e = prim_max(p.stream, in, count, dmax);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host_out, dmax, sizeof(int), cudaMemcpyDeviceToHost, p.stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(p.stream);
    cudaFreeAsync(dmax, p.stream);
    return e;
}

#define LPM_TRY(x)                                                                                                     \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess)                                                                                         \
            return e_;                                                                                                 \
    } while (0)

cudaError_t build_topology(Problem &p, const double *xyz_host, int *err_code)
{
    const int n = p.n;
    *err_code = 0;
    const bool user_bonds = p.desc.bond_nb0 && p.desc.bond_nb1 && p.desc.bond_p2;
    // grid of cells no smaller than the largest search radius
    const double rc0 = 1.01 * p.cell.cutoff[0], rc1 = 1.01 * p.cell.cutoff[1];
    Grid g;
    double hi[3];
    for (int k = 0; k < 3; ++k)
    {
        g.lo[k] = 1e300;
        hi[k] = -1e300;
    }
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k)
        {
            g.lo[k] = std::min(g.lo[k], xyz_host[3 * i + k]);
            hi[k] = std::max(hi[k], xyz_host[3 * i + k]);
        }
    g.h = rc1 * 1.0001;
    int64_t ncell = 1;
    for (int k = 0; k < 3; ++k)
    {
        double span = (hi[k] - g.lo[k]) / g.h;
        g.nc[k] = (int)std::min(std::floor(span) + 1.0, 4096.0);
        if (g.nc[k] < 1)
            g.nc[k] = 1;
        ncell *= g.nc[k];
    }
    while (ncell > 64ll * 1024 * 1024)
    { // very sparse clouds: coarser cells keep the grid bounded (still exact, only slower)
        g.h *= 2;
        ncell = 1;
        for (int k = 0; k < 3; ++k)
        {
            g.nc[k] = (int)std::floor((hi[k] - g.lo[k]) / g.h) + 1;
            ncell *= g.nc[k];
        }
    }

    int *key = nullptr, *ids = nullptr, *skey = nullptr, *sid = nullptr, *cbeg = nullptr, *cend = nullptr;
    LPM_TRY(cudaMallocAsync(&key, sizeof(int) * n, p.stream));
    LPM_TRY(cudaMallocAsync(&ids, sizeof(int) * n, p.stream));
    LPM_TRY(cudaMallocAsync(&skey, sizeof(int) * n, p.stream));
    LPM_TRY(cudaMallocAsync(&sid, sizeof(int) * n, p.stream));
    LPM_TRY(cudaMallocAsync(&cbeg, sizeof(int) * ncell, p.stream));
    LPM_TRY(cudaMallocAsync(&cend, sizeof(int) * ncell, p.stream));
    LPM_TRY(cudaMemsetAsync(cbeg, 0, sizeof(int) * ncell, p.stream));
    LPM_TRY(cudaMemsetAsync(cend, 0, sizeof(int) * ncell, p.stream));
    const int T = 256;
    k_cell_keys<<<div_up(n, T), T, 0, p.stream>>>(n, p.xyz, g, key, ids);
    {
        LPM_TRY(prim_sort_pairs(p.stream, key, ids, skey, sid, n));
    }
    k_cell_bounds<<<div_up(n, T), T, 0, p.stream>>>(n, skey, cbeg, cend);

    int *pad_id = nullptr;
    double *pad_d = nullptr;
    LPM_TRY(cudaMallocAsync(&pad_id, sizeof(int) * (size_t)n * kMaxBonds, p.stream));
    LPM_TRY(cudaMallocAsync(&pad_d, sizeof(double) * (size_t)n * kMaxBonds, p.stream));
    LPM_TRY(dalloc(p, &p.nb, n));
    LPM_TRY(dalloc(p, &p.nb0, n));
    LPM_TRY(dalloc(p, &p.bstart, (size_t)n + 1));
    if (user_bonds)
    {
        // caller-supplied lists (bond file / pre-crack): padded copy, distances computed here
        std::vector<int> hnb(n), hnb0(n), hpad((size_t)n * kMaxBonds, 0);
        size_t o = 0;
        for (int i = 0; i < n; ++i)
        {
            const int a0 = p.desc.bond_nb0[i], a1 = p.desc.bond_nb1[i];
            if (a0 < 0 || a1 < 0 || a0 + a1 > kMaxBonds)
            {
                *err_code = LPMGPU_ERR_TOPOLOGY;
                return cudaSuccess;
            }
            hnb0[i] = a0;
            hnb[i] = a0 + a1;
            for (int q = 0; q < a0 + a1; ++q)
            {
                const int j = p.desc.bond_p2[o++];
                if (j < 0 || j >= n || j == i)
                {
                    *err_code = LPMGPU_ERR_TOPOLOGY;
                    return cudaSuccess;
                }
                hpad[(size_t)i * kMaxBonds + q] = j;
            }
        }
        LPM_TRY(cudaMemcpyAsync(p.nb, hnb.data(), sizeof(int) * n, cudaMemcpyHostToDevice, p.stream));
        LPM_TRY(cudaMemcpyAsync(p.nb0, hnb0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, p.stream));
        LPM_TRY(cudaMemcpyAsync(pad_id, hpad.data(), sizeof(int) * hpad.size(), cudaMemcpyHostToDevice, p.stream));
        k_bonds_dist<<<div_up(n, 128), 128, 0, p.stream>>>(n, p.xyz, pad_id, p.nb, pad_d);
        LPM_TRY(cudaStreamSynchronize(p.stream)); // the host vectors above must outlive the copies
    }
    else
        k_bonds_find<<<div_up(n, 128), 128, 0, p.stream>>>(n, p.xyz, g, sid, cbeg, cend, rc0, rc1, pad_id, pad_d,
                                                           p.nb, p.nb0, p.scal);
    LPM_TRY(cudaGetLastError());
    // bstart = exclusive scan of nb (n+1 entries: the appended zero yields the total)
    int *nbx = nullptr;
    LPM_TRY(cudaMallocAsync(&nbx, sizeof(int) * ((size_t)n + 1), p.stream));
    LPM_TRY(cudaMemsetAsync(nbx, 0, sizeof(int) * ((size_t)n + 1), p.stream));
    LPM_TRY(cudaMemcpyAsync(nbx, p.nb, sizeof(int) * n, cudaMemcpyDeviceToDevice, p.stream));
    LPM_TRY(exclusive_scan(p, nbx, p.bstart, n + 1));
    int nbonds = 0;
    LPM_TRY(cudaMemcpyAsync(&nbonds, p.bstart + n, sizeof(int), cudaMemcpyDeviceToHost, p.stream));
    LPM_TRY(cudaMemcpyAsync(p.scal_host, p.scal, sizeof(Scalars), cudaMemcpyDeviceToHost, p.stream));
    LPM_TRY(cudaStreamSynchronize(p.stream));
    if (p.scal_host->err)
    {
        *err_code = LPMGPU_ERR_TOPOLOGY;
        return cudaSuccess;
    }
    p.nbonds = nbonds;
    const size_t nb = (size_t)nbonds;
    LPM_TRY(dalloc(p, &p.bp2, nb));
    LPM_TRY(dalloc(p, &p.brev, nb));
    LPM_TRY(dalloc(p, &p.dis0, nb));
    LPM_TRY(dalloc(p, &p.dis, nb));
    LPM_TRY(dalloc(p, &p.dis_last, nb));
    LPM_TRY(dalloc(p, &p.dLe, nb));
    LPM_TRY(dalloc(p, &p.dLp, nb));
    LPM_TRY(dalloc(p, &p.dLp_last, nb));
    LPM_TRY(dalloc(p, &p.bstrain, nb));
    LPM_TRY(dalloc(p, &p.Kn, nb));
    LPM_TRY(dalloc(p, &p.Tv, nb));
    LPM_TRY(dalloc(p, &p.cs, 3 * nb));
    LPM_TRY(dalloc(p, &p.bforce, nb));
    LPM_TRY(dalloc(p, &p.bforce_last, nb));
    LPM_TRY(dalloc(p, &p.bdamage, nb));
    LPM_TRY(dalloc(p, &p.bdamage_last, nb));
    k_bonds_fill<<<div_up(n, T), T, 0, p.stream>>>(n, p.xyz, pad_id, pad_d, p.nb, p.nb0, p.bstart,
                                                   p.cell.lattice == LPMGPU_HEXAGON2D, p.kntv[0], p.kntv[1],
                                                   p.kntv[2], p.bp2, p.dis0, p.dis, p.dis_last, p.cs, p.Kn, p.Tv);
    k_bonds_rev<<<div_up(n, T), T, 0, p.stream>>>(n, p.bstart, p.nb0, p.bp2, p.brev, p.scal);
    LPM_TRY(cudaGetLastError());
    if (p.desc.bond_kn)
        LPM_TRY(cudaMemcpyAsync(p.Kn, p.desc.bond_kn, sizeof(double) * nb, cudaMemcpyHostToDevice, p.stream));
    if (p.desc.bond_tv)
        LPM_TRY(cudaMemcpyAsync(p.Tv, p.desc.bond_tv, sizeof(double) * nb, cudaMemcpyHostToDevice, p.stream));
    if (p.desc.bond_damage)
    {
        LPM_TRY(cudaMemcpyAsync(p.bdamage, p.desc.bond_damage, sizeof(double) * nb, cudaMemcpyHostToDevice, p.stream));
        LPM_TRY(cudaMemcpyAsync(p.bdamage_last, p.desc.bond_damage, sizeof(double) * nb, cudaMemcpyHostToDevice,
                                p.stream));
    }
    cudaFreeAsync(pad_id, p.stream);
    cudaFreeAsync(pad_d, p.stream);
    cudaFreeAsync(key, p.stream);
    cudaFreeAsync(ids, p.stream);
    cudaFreeAsync(skey, p.stream);
    cudaFreeAsync(sid, p.stream);
    cudaFreeAsync(cbeg, p.stream);
    cudaFreeAsync(cend, p.stream);

    // connections
    int *pad_c = nullptr, *ncx = nullptr;
    LPM_TRY(cudaMallocAsync(&pad_c, sizeof(int) * (size_t)n * kMaxConns, p.stream));
    LPM_TRY(cudaMallocAsync(&ncx, sizeof(int) * ((size_t)n + 1), p.stream));
    LPM_TRY(cudaMemsetAsync(ncx, 0, sizeof(int) * ((size_t)n + 1), p.stream));
    LPM_TRY(dalloc(p, &p.nlq, n));
    LPM_TRY(dalloc(p, &p.cstart, (size_t)n + 1));
    {
        const int warps = 8;
        size_t smem = sizeof(int) * kMaxCand * warps;
        k_conns<<<div_up(n, warps), warps * 32, smem, p.stream>>>(n, p.bstart, p.nb0, p.bp2, pad_c, ncx, p.nlq,
                                                                   p.scal);
        LPM_TRY(cudaGetLastError());
    }
    LPM_TRY(exclusive_scan(p, ncx, p.cstart, n + 1));
    int nnzb = 0;
    LPM_TRY(cudaMemcpyAsync(&nnzb, p.cstart + n, sizeof(int), cudaMemcpyDeviceToHost, p.stream));
    LPM_TRY(cudaMemcpyAsync(p.scal_host, p.scal, sizeof(Scalars), cudaMemcpyDeviceToHost, p.stream));
    LPM_TRY(cudaStreamSynchronize(p.stream));
    if (p.scal_host->err)
    {
        *err_code = LPMGPU_ERR_TOPOLOGY;
        return cudaSuccess;
    }
    p.nnzb = nnzb;
    LPM_TRY(dalloc(p, &p.conns, (size_t)nnzb));
    k_conns_fill<<<n, 64, 0, p.stream>>>(n, pad_c, p.cstart, p.conns);
    LPM_TRY(cudaGetLastError());
    LPM_TRY(reduce_max(p, ncx, n, &p.max_conns));
    LPM_TRY(reduce_max(p, p.nb, n, &p.max_bonds));
    k_records<<<div_up(n, T), T, 0, p.stream>>>(n, p.bstart, p.nb0, p.bp2, ncx);
    LPM_TRY(reduce_max(p, ncx, n, &p.max_records));
    cudaFreeAsync(pad_c, p.stream);
    cudaFreeAsync(ncx, p.stream);

    // sliced-ELL layout: rows by descending connection count (stable sort), slices of 32; in 2D
    // each slice width spread over the slice order
    {
        int *key = nullptr, *ids = nullptr, *skey = nullptr;
        LPM_TRY(cudaMallocAsync(&key, sizeof(int) * n, p.stream));
        LPM_TRY(cudaMallocAsync(&ids, sizeof(int) * n, p.stream));
        LPM_TRY(cudaMallocAsync(&skey, sizeof(int) * n, p.stream));
        LPM_TRY(dalloc(p, &p.perm, n));
        LPM_TRY(dalloc(p, &p.iperm, n));
        k_sell_keys<<<div_up(n, T), T, 0, p.stream>>>(n, p.cstart, key, ids);
        LPM_TRY(prim_sort_pairs(p.stream, key, ids, skey, p.perm, n));
        p.nslices = div_up(n, kSlice);
        int64_t *width = nullptr;
        LPM_TRY(cudaMallocAsync(&width, sizeof(int64_t) * (p.nslices + 1), p.stream));
        LPM_TRY(dalloc(p, &p.slice_off, (size_t)p.nslices + 1));
        k_sell_width<<<div_up(p.nslices + 1, T), T, 0, p.stream>>>(n, p.nslices, p.perm, p.cstart, nullptr, width);
        LPM_TRY(cudaGetLastError());
        if (p.dim == 2)
            LPM_TRY(spread_slices(p, width));
        LPM_TRY(exclusive_scan(p, width, p.slice_off, p.nslices + 1));
        LPM_TRY(cudaMemcpyAsync(&p.nsb, p.slice_off + p.nslices, sizeof(int64_t), cudaMemcpyDeviceToHost, p.stream));
        LPM_TRY(cudaStreamSynchronize(p.stream));
        LPM_TRY(dalloc(p, &p.col_sell, (size_t)p.nsb * kSlice));
        k_sell_fill<<<div_up((int64_t)p.nslices * kSlice, T), T, 0, p.stream>>>(n, p.nslices, p.perm, p.cstart,
                                                                                p.conns, p.slice_off, p.iperm,
                                                                                p.col_sell);
        LPM_TRY(cudaGetLastError());
        cudaFreeAsync(width, p.stream);
        cudaFreeAsync(key, p.stream);
        cudaFreeAsync(ids, p.stream);
        cudaFreeAsync(skey, p.stream);
    }

    // reference K_pointer
    int64_t *kv = nullptr;
    LPM_TRY(cudaMallocAsync(&kv, sizeof(int64_t) * ((size_t)n + 1), p.stream));
    LPM_TRY(dalloc(p, &p.kp_ref, (size_t)n + 1));
    k_kp_counts<<<div_up(n + 1, T), T, 0, p.stream>>>(n, p.dim, p.nlq, kv);
    LPM_TRY(exclusive_scan(p, kv, p.kp_ref, n + 1));
    LPM_TRY(cudaMemcpyAsync(&p.nnz_upper, p.kp_ref + n, sizeof(int64_t), cudaMemcpyDeviceToHost, p.stream));
    LPM_TRY(cudaStreamSynchronize(p.stream));
    cudaFreeAsync(kv, p.stream);
    return cudaSuccess;
}

} // namespace lpm
