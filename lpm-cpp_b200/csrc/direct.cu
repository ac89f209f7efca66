// Direct solve of the Newton system: the device counterpart of Solver::LPM_PARDISO
// (include/solver.h:191-274), which the reference's SolverMode::PARDISO runs in place of its CG.
//
//   * Ordering (host, once per problem): reverse Cuthill-McKee over the particle connection graph
//     (the conns of assembly.h:237-266) narrows the band; particle i's unknowns become
//     d * rank(i) + r.  The half-bandwidth is kd = d * max |rank(i) - rank(j)| over connected
//     pairs + d - 1.
//   * Band fill (device): the BC-eliminated stiffness, read from its sliced-ELL blocks, into the
//     permuted lower band (band_chol.cuh's layout).
//   * Factorisation (device, once per assembled K: K is fixed through a load step's Newton
//     iterations, solver_static.h:107-118): blocked band Cholesky in column blocks of kBandNB,
//     three kernels per block (diagonal block, rows below it, trailing window).
//   * Solve (device, every Newton iteration): forward and backward substitution on the factor.
// The band costs n * (kd + 1) doubles; 2D plates fit easily, wide 3D bands are rejected with
// LPMGPU_ERR_OUT_OF_MEMORY before anything is allocated.  A pivot that is not positive (a
// singular or indefinite K, e.g. a particle left without bonds) is LPMGPU_ERR_NOT_SPD.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "band_chol.cuh"
#include "lpm_internal.cuh"

namespace lpm
{

constexpr int kBandNB = 32;                       // column block of the factorisation and solves
constexpr int64_t kBandMaxBytes = int64_t(32) << 30; // band storage limit per problem (32 GiB)

// Reverse Cuthill-McKee over a graph in CSR (rows ascending ids, self loops allowed): rank[i] is
// i's position.  Each connected component starts at a pseudo-peripheral vertex (the last vertex
// reached by two breadth-first sweeps from its lowest-degree vertex); neighbours join in
// ascending degree, then id.  When the given order (the identity) has a band at most as wide,
// it is kept instead.  Returns the largest |rank(i) - rank(j)| over the edges.
int64_t rcm_order(int n, const int *start, const int *adj, int *rank)
{
    std::vector<int> deg(n), order;
    order.reserve(n);
    for (int i = 0; i < n; ++i)
        deg[i] = start[i + 1] - start[i];
    std::vector<char> seen(n, 0);
    std::vector<int> level(n, -1), byid(n);
    for (int i = 0; i < n; ++i)
        byid[i] = i;
    std::stable_sort(byid.begin(), byid.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    auto bfs_last = [&](int s) {
        // the last vertex of a breadth-first sweep from s inside its component
        std::vector<int> q{s};
        level[s] = 0;
        size_t h = 0;
        int last = s;
        while (h < q.size())
        {
            const int v = q[h++];
            last = v;
            for (int k = start[v]; k < start[v + 1]; ++k)
                if (level[adj[k]] < 0)
                {
                    level[adj[k]] = level[v] + 1;
                    q.push_back(adj[k]);
                }
        }
        for (int v : q)
            level[v] = -1;
        return last;
    };
    std::vector<int> nb;
    for (int s0 : byid)
    {
        if (seen[s0])
            continue;
        const int s = bfs_last(bfs_last(s0));
        size_t h = order.size();
        order.push_back(s);
        seen[s] = 1;
        while (h < order.size())
        {
            const int v = order[h++];
            nb.clear();
            for (int k = start[v]; k < start[v + 1]; ++k)
                if (!seen[adj[k]])
                {
                    seen[adj[k]] = 1;
                    nb.push_back(adj[k]);
                }
            std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
            order.insert(order.end(), nb.begin(), nb.end());
        }
    }
    for (int p = 0; p < n; ++p)
        rank[order[n - 1 - p]] = p; // reversed
    int64_t bw = 0, bw_id = 0;
    for (int i = 0; i < n; ++i)
        for (int k = start[i]; k < start[i + 1]; ++k)
        {
            bw = std::max<int64_t>(bw, std::abs((int64_t)rank[i] - rank[adj[k]]));
            bw_id = std::max<int64_t>(bw_id, std::abs((int64_t)i - adj[k]));
        }
    // the lattice generators' own order (row by row along the longest side) is often as narrow:
    // keep whichever band is narrower
    if (bw_id <= bw)
    {
        for (int i = 0; i < n; ++i)
            rank[i] = i;
        bw = bw_id;
    }
    return bw;
}

// One thread per particle i: its stiffness block row (sliced ELL, BCs eliminated) into the
// permuted lower band, entries on or below the diagonal only; the full symmetric storage holds
// every lower entry exactly once.
template <int D>
__global__ void k_band_fill(int n, const int *__restrict__ rowptr, const int *__restrict__ iperm_sell,
                            const int64_t *__restrict__ slice_off, const int *__restrict__ col_sell,
                            const double *__restrict__ K, const int *__restrict__ rank, int64_t ldab,
                            double *__restrict__ AB)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int pos = iperm_sell[i], s = pos / kSlice, l = pos % kSlice;
    const int nc = rowptr[i + 1] - rowptr[i];
    const int64_t ri = (int64_t)D * rank[i];
    for (int k = 0; k < nc; ++k)
    {
        const int64_t b = slice_off[s] + k;
        const int j = col_sell[b * kSlice + l];
        const int64_t cj = (int64_t)D * rank[j];
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c)
            {
                const int64_t R = ri + r, C = cj + c;
                if (R >= C)
                    AB[(R - C) + C * ldab] = K[(b * D * D + r * D + c) * kSlice + l];
            }
    }
}

// The diagonal block by one warp: the block's lower triangle (inside the band) staged in shared
// memory, lane i owning row i.  Per column jj: the pivot's square root, the column scaled, the
// trailing entries updated, each entry receiving exactly the operations, in the order, of
// band::potrf_block (which the host tests run), so the factor is bit for bit the same.
__global__ void __launch_bounds__(32) k_potrf(double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, int *fail)
{
    __shared__ double a[32][33];
    __shared__ int bad;
    const int i = threadIdx.x;
    if (i == 0)
        bad = 0;
    if (i < jb)
        for (int j = 0; j <= i; ++j)
            a[i][j] = (i - j <= kd) ? band::at(AB, ldab, j0 + i, j0 + j) : 0.0;
    __syncwarp();
    for (int jj = 0; jj < jb; ++jj)
    {
        if (i == jj)
        {
            const double v = a[jj][jj];
            if (!(v > 0.0))
                bad = jj + 1;
            else
                a[jj][jj] = sqrt(v);
        }
        __syncwarp();
        if (bad)
            break;
        const double d = a[jj][jj];
        if (i > jj && i < jb && i - jj <= kd)
            a[i][jj] = a[i][jj] / d;
        __syncwarp();
        // row i: entries (i, c), jj < c <= i, in ascending c as the one-thread loop reaches them
        if (i > jj && i < jb && i - jj <= kd)
            for (int c = jj + 1; c <= i; ++c)
                if (c - jj <= kd)
                    a[i][c] = a[i][c] - a[i][jj] * a[c][jj];
        __syncwarp();
    }
    if (bad)
    {
        if (i == 0 && *fail == 0)
            *fail = (int)(j0 + bad);
        return;
    }
    if (i < jb)
        for (int j = 0; j <= i; ++j)
            if (i - j <= kd)
                band::at(AB, ldab, j0 + i, j0 + j) = a[i][j];
}

// The rows below the diagonal block, one thread per row, with the factored block and the thread's
// row staged in shared memory; each entry gets band::trsm_row's operations in its order.
constexpr int kTrsmThreads = 128;
__global__ void __launch_bounds__(kTrsmThreads) k_trsm(double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb,
                                                       int64_t m2)
{
    __shared__ double L[32][33];
    __shared__ double row[kTrsmThreads][33];
    for (int q = threadIdx.x; q < 32 * 32; q += blockDim.x)
    {
        const int r = q / 32, c = q % 32;
        L[r][c] = (r < jb && c <= r && r - c <= kd) ? band::at(AB, ldab, j0 + r, j0 + c) : 0.0;
    }
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t i = j0 + jb + t;
    double *w = row[threadIdx.x];
    if (t < m2)
        for (int jj = 0; jj < jb; ++jj)
            w[jj] = (i - (j0 + jj) <= kd) ? band::at(AB, ldab, i, j0 + jj) : 0.0;
    __syncthreads();
    if (t >= m2)
        return;
    for (int jj = 0; jj < jb; ++jj)
    {
        const int64_t j = j0 + jj;
        if (i - j > kd)
            continue;
        double v = w[jj];
        for (int kk = 0; kk < jj; ++kk)
            if (i - (j0 + kk) <= kd)
                v = v - w[kk] * L[jj][kk];
        v = v / L[jj][jj];
        w[jj] = v;
        band::at(AB, ldab, i, j) = v;
    }
}

// threads along i (contiguous band columns), blocks along c
__global__ void k_syrk(double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, int64_t m2)
{
    const int64_t c0 = j0 + jb, e = c0 + m2;
    for (int64_t cy = blockIdx.y; cy < m2; cy += gridDim.y)
    {
        const int64_t c = c0 + cy;
        const int64_t i = c + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (i < e && i - c <= kd)
            band::syrk_entry(AB, ldab, kd, j0, jb, i, c);
    }
}

__global__ void k_fwd_block(const double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, double *y)
{
    band::fwd_block(AB, ldab, kd, j0, jb, y);
}

__global__ void k_fwd_update(const double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, int64_t m2, double *y)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m2)
        band::fwd_update_row(AB, ldab, kd, j0, jb, j0 + jb + t, y);
}

__global__ void k_bwd_update(const double *AB, int64_t ldab, int64_t kd, int64_t n, int64_t j0, int64_t jb, double *y)
{
    const int64_t t = threadIdx.x;
    if (t < jb)
        band::bwd_update_col(AB, ldab, kd, n, j0, jb, j0 + t, y);
}

__global__ void k_bwd_block(const double *AB, int64_t ldab, int64_t kd, int64_t j0, int64_t jb, double *y)
{
    band::bwd_block(AB, ldab, kd, j0, jb, y);
}

// y[d*rank(i)+r] = src[d*i+r]  /  dst[d*i+r] = y[d*rank(i)+r]
__global__ void k_band_perm(int n, int dim, const int *__restrict__ rank, const double *__restrict__ src,
                            double *__restrict__ dst, int inverse)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (int64_t)n * dim)
        return;
    const int i = (int)(q / dim), r = (int)(q % dim);
    const int64_t pq = (int64_t)dim * rank[i] + r;
    if (inverse)
        dst[q] = src[pq];
    else
        dst[pq] = src[q];
}

// The ordering, the band's size and its storage; once per problem.
static int32_t direct_setup(Problem &p)
{
    if (p.band_ab)
        return LPMGPU_OK;
    const int n = p.n;
    std::vector<int> start((size_t)n + 1), adj((size_t)p.nnzb), rank(n);
    cudaError_t e = cudaMemcpyAsync(start.data(), p.cstart, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost,
                                    p.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(adj.data(), p.conns, sizeof(int) * (size_t)p.nnzb, cudaMemcpyDeviceToHost, p.stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(p.stream);
    if (e != cudaSuccess)
    {
        set_last_error(std::string("direct solver set-up: ") + cudaGetErrorString(e));
        return LPMGPU_ERR_CUDA;
    }
    const int64_t bw = rcm_order(n, start.data(), adj.data(), rank.data());
    const int64_t ndof = (int64_t)n * p.dim;
    const int64_t kd = std::min<int64_t>((int64_t)p.dim * bw + p.dim - 1, ndof - 1);
    const int64_t ldab = kd + 1;
    if (ldab * ndof * (int64_t)sizeof(double) > kBandMaxBytes)
    {
        set_last_error("direct solver: the band (" + std::to_string(ndof) + " unknowns, half-bandwidth " +
                       std::to_string(kd) + ") is larger than the 32 GiB the solver allows; use the CG");
        return LPMGPU_ERR_OUT_OF_MEMORY;
    }
    if ((e = dalloc(p, &p.band_rank, (size_t)n)) != cudaSuccess ||
        (e = dalloc(p, &p.band_y, (size_t)ndof)) != cudaSuccess ||
        (e = dalloc(p, &p.band_fail, 1)) != cudaSuccess ||
        (e = dalloc(p, &p.band_ab, (size_t)(ldab * ndof))) != cudaSuccess)
    {
        (void)cudaGetLastError(); // a failed allocation is reported here, not by a later launch check
        p.band_ab = nullptr;
        set_last_error(std::string("direct solver: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? LPMGPU_ERR_OUT_OF_MEMORY : LPMGPU_ERR_CUDA;
    }
    if ((e = cudaMemcpyAsync(p.band_rank, rank.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, p.stream)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(p.stream)) != cudaSuccess)
        return LPMGPU_ERR_CUDA;
    p.band_kd = kd;
    p.band_factored = -1;
    return LPMGPU_OK;
}

// Band fill + blocked factorisation of the current K.
template <int D>
static cudaError_t factor(Problem &p)
{
    const int64_t ndof = (int64_t)p.n * D, kd = p.band_kd, ldab = kd + 1;
    cudaError_t e = cudaMemsetAsync(p.band_ab, 0, sizeof(double) * (size_t)(ldab * ndof), p.stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(p.band_fail, 0, sizeof(int), p.stream);
    if (e != cudaSuccess)
        return e;
    k_band_fill<D><<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.cstart, p.iperm, p.slice_off, p.col_sell, p.K,
                                                          p.band_rank, ldab, p.band_ab);
    p.ctr.kernel_launches++;
    for (int64_t j0 = 0; j0 < ndof; j0 += kBandNB)
    {
        const int64_t jb = std::min<int64_t>(kBandNB, ndof - j0);
        const int64_t m2 = band::below_end(ndof, kd, j0, jb) - (j0 + jb);
        k_potrf<<<1, 32, 0, p.stream>>>(p.band_ab, ldab, kd, j0, jb, p.band_fail);
        p.ctr.kernel_launches++;
        if (m2 > 0)
        {
            k_trsm<<<(unsigned)div_up(m2, 128), 128, 0, p.stream>>>(p.band_ab, ldab, kd, j0, jb, m2);
            const dim3 grid((unsigned)div_up(m2, 128), (unsigned)std::min<int64_t>(m2, 65535));
            k_syrk<<<grid, 128, 0, p.stream>>>(p.band_ab, ldab, kd, j0, jb, m2);
            p.ctr.kernel_launches += 2;
        }
    }
    return cudaGetLastError();
}

// Forward and backward substitution of p.res into p.x.
template <int D>
static cudaError_t substitute(Problem &p)
{
    const int64_t ndof = (int64_t)p.n * D, kd = p.band_kd, ldab = kd + 1;
    const int nb = (int)div_up(ndof, 256);
    k_band_perm<<<nb, 256, 0, p.stream>>>(p.n, D, p.band_rank, p.res, p.band_y, 0);
    p.ctr.kernel_launches++;
    for (int64_t j0 = 0; j0 < ndof; j0 += kBandNB)
    {
        const int64_t jb = std::min<int64_t>(kBandNB, ndof - j0);
        const int64_t m2 = band::below_end(ndof, kd, j0, jb) - (j0 + jb);
        k_fwd_block<<<1, 1, 0, p.stream>>>(p.band_ab, ldab, kd, j0, jb, p.band_y);
        p.ctr.kernel_launches++;
        if (m2 > 0)
        {
            k_fwd_update<<<(unsigned)div_up(m2, 128), 128, 0, p.stream>>>(p.band_ab, ldab, kd, j0, jb, m2, p.band_y);
            p.ctr.kernel_launches++;
        }
    }
    const int64_t last = ((ndof - 1) / kBandNB) * kBandNB;
    for (int64_t j0 = last; j0 >= 0; j0 -= kBandNB)
    {
        const int64_t jb = std::min<int64_t>(kBandNB, ndof - j0);
        if (j0 + jb < ndof)
        {
            k_bwd_update<<<1, kBandNB, 0, p.stream>>>(p.band_ab, ldab, kd, ndof, j0, jb, p.band_y);
            p.ctr.kernel_launches++;
        }
        k_bwd_block<<<1, 1, 0, p.stream>>>(p.band_ab, ldab, kd, j0, jb, p.band_y);
        p.ctr.kernel_launches++;
    }
    k_band_perm<<<nb, 256, 0, p.stream>>>(p.n, D, p.band_rank, p.band_y, p.x, 1);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// K x = res into p.x by the band Cholesky; the factor is reused while K is unchanged.
int32_t solve_direct(Problem &p)
{
    int32_t s = direct_setup(p);
    if (s != LPMGPU_OK)
        return s;
    cudaError_t e = cudaSuccess;
    if (p.band_factored != p.k_version)
    {
        e = p.dim == 2 ? factor<2>(p) : factor<3>(p);
        int fail = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&fail, p.band_fail, sizeof(int), cudaMemcpyDeviceToHost, p.stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(p.stream);
        if (e != cudaSuccess)
        {
            set_last_error(std::string("direct solver: ") + cudaGetErrorString(e));
            return LPMGPU_ERR_CUDA;
        }
        if (fail)
        {
            p.band_factored = -1;
            set_last_error("direct solver: the stiffness is not positive definite (pivot " + std::to_string(fail) +
                           " of the reordered system)");
            return LPMGPU_ERR_NOT_SPD;
        }
        p.band_factored = p.k_version;
    }
    e = p.dim == 2 ? substitute<2>(p) : substitute<3>(p);
    if (e != cudaSuccess)
    {
        set_last_error(std::string("direct solver: ") + cudaGetErrorString(e));
        return LPMGPU_ERR_CUDA;
    }
    return LPMGPU_OK;
}

} // namespace lpm

extern "C" int32_t lpmgpu_band_order(int32_t n, const int32_t *start, const int32_t *adj, int32_t *rank,
                                     int64_t *bandwidth)
{
    if (n <= 0 || !start || !adj || !rank || !bandwidth || start[0] != 0)
        return LPMGPU_ERR_INVALID_ARG;
    for (int i = 0; i < n; ++i)
        if (start[i + 1] < start[i])
            return LPMGPU_ERR_INVALID_ARG;
    for (int k = 0; k < start[n]; ++k)
        if (adj[k] < 0 || adj[k] >= n)
            return LPMGPU_ERR_INVALID_ARG;
    *bandwidth = lpm::rcm_order(n, start, adj, rank);
    return LPMGPU_OK;
}
