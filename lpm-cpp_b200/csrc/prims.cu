// Device-wide primitives of the set-up paths (topology, sliced-ELL layout, nonlocal lists):
// exclusive scans, a maximum, a stable key/value sort and a segmented sort.  They run once per
// problem, so they favour simple, deterministic forms over peak speed:
//   * scan: per-tile sums, one block scanning the tile sums, per-tile scans with their offsets;
//   * maximum: one block, fixed-order reduction;
//   * sorts: a bitonic network over 64-bit composite keys (key << 32 | position, or segment << 32
//     | value), so equal keys keep their input order (stable) and segments stay apart; stages
//     whose partner distance fits a 4096-key tile run in shared memory.
#include "lpm_internal.cuh"

#include <climits>

namespace lpm
{

namespace
{

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems; // elements per tile
constexpr int kSortTile = 4096;                      // keys per shared-memory bitonic tile
constexpr int kSortThreads = 1024;

// exclusive scan of the kScanThreads values v within a block (fixed order); returns the total
template <typename T>
__device__ T block_exclusive(T &v, T *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
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
        T t = lane < nw ? sh[lane] : T(0);
        for (int o = 1; o < 32; o <<= 1)
        {
            const T y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o)
                t += y;
        }
        sh[lane] = t;
    }
    __syncthreads();
    const T before = (w > 0 ? sh[w - 1] : T(0)) + x - v;
    const T total = sh[nw - 1];
    __syncthreads();
    v = before;
    return total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const T *__restrict__ in, int64_t count, T *__restrict__ sums)
{
    __shared__ T sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    T s = 0;
    for (int k = 0; k < kScanItems; ++k)
    {
        const int64_t q = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (q < count)
            s += in[q];
    }
    T v = s;
    const T tot = block_exclusive(v, sh);
    if (threadIdx.x == 0)
        sums[blockIdx.x] = tot;
}

// exclusive scan of v[0 .. n) into out[0 .. n) by one block (chunks of consecutive entries)
template <typename T>
__global__ void __launch_bounds__(1024) k_scan_one_block(const T *__restrict__ v, int64_t n, T *__restrict__ out)
{
    __shared__ T sh[32];
    const int64_t chunk = (n + blockDim.x - 1) / blockDim.x;
    const int64_t lo = min(n, (int64_t)threadIdx.x * chunk), hi = min(n, lo + chunk);
    T s = 0;
    for (int64_t k = lo; k < hi; ++k)
        s += v[k];
    T run = s;
    block_exclusive(run, sh);
    for (int64_t k = lo; k < hi; ++k)
    {
        const T x = v[k];
        out[k] = run;
        run += x;
    }
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const T *__restrict__ in, int64_t count,
                                                          const T *__restrict__ offs, T *__restrict__ out)
{
    __shared__ T tile[kScanTile];
    __shared__ T sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    for (int k = 0; k < kScanItems; ++k)
    {
        const int64_t q = base + (int64_t)k * kScanThreads + threadIdx.x;
        tile[k * kScanThreads + threadIdx.x] = q < count ? in[q] : T(0);
    }
    __syncthreads();
    T loc[kScanItems];
    T s = 0;
    for (int k = 0; k < kScanItems; ++k)
    {
        loc[k] = s;
        s += tile[threadIdx.x * kScanItems + k];
    }
    T v = s;
    block_exclusive(v, sh);
    const T off = offs[blockIdx.x] + v;
    for (int k = 0; k < kScanItems; ++k)
        tile[threadIdx.x * kScanItems + k] = off + loc[k];
    __syncthreads();
    for (int k = 0; k < kScanItems; ++k)
    {
        const int64_t q = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (q < count)
            out[q] = tile[k * kScanThreads + threadIdx.x];
    }
}

template <typename T>
cudaError_t scan_impl(cudaStream_t st, const T *in, T *out, int64_t count)
{
    if (count <= 0)
        return cudaSuccess;
    const int64_t tiles = (count + kScanTile - 1) / kScanTile;
    T *sums = nullptr, *offs = nullptr;
    cudaError_t e = cudaMallocAsync(&sums, sizeof(T) * 2 * tiles, st);
    if (e != cudaSuccess)
        return e;
    offs = sums + tiles;
    k_tile_sums<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, count, sums);
    k_scan_one_block<T><<<1, 1024, 0, st>>>(sums, tiles, offs);
    k_tile_scan<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, count, offs, out);
    e = cudaGetLastError();
    cudaFreeAsync(sums, st);
    return e;
}

__global__ void __launch_bounds__(1024) k_max_one_block(const int *__restrict__ in, int64_t count, int *__restrict__ out)
{
    __shared__ int sh[32];
    int m = INT_MIN;
    for (int64_t q = threadIdx.x; q < count; q += blockDim.x)
        m = max(m, in[q]);
    for (int o = 16; o > 0; o >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        int t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : INT_MIN;
        for (int o = 16; o > 0; o >>= 1)
            t = max(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0)
            *out = t;
    }
}

// ---- bitonic network over N = 2^k 64-bit keys (ascending)
__device__ __forceinline__ void cas(unsigned long long &a, unsigned long long &b, bool up)
{
    if ((a > b) == up)
    {
        const unsigned long long t = a;
        a = b;
        b = t;
    }
}

// all stages k = 2 .. kSortTile inside each tile
__global__ void __launch_bounds__(kSortThreads) k_bitonic_tile_full(unsigned long long *__restrict__ keys)
{
    __shared__ unsigned long long t[kSortTile];
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int q = threadIdx.x; q < kSortTile; q += blockDim.x)
        t[q] = keys[base + q];
    __syncthreads();
    for (int k = 2; k <= kSortTile; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int q = threadIdx.x; q < kSortTile / 2; q += blockDim.x)
            {
                const int i = 2 * q - (q & (j - 1)); // the lower index of the q-th pair at distance j
                const int64_t gi = base + i;
                cas(t[i], t[i + j], (gi & k) == 0);
            }
            __syncthreads();
        }
    for (int q = threadIdx.x; q < kSortTile; q += blockDim.x)
        keys[base + q] = t[q];
}

// the stages j = j0, j0/2, .., 1 of merge size k, inside each tile (j0 < kSortTile)
__global__ void __launch_bounds__(kSortThreads) k_bitonic_tile_merge(unsigned long long *__restrict__ keys, int64_t k,
                                                                     int j0)
{
    __shared__ unsigned long long t[kSortTile];
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int q = threadIdx.x; q < kSortTile; q += blockDim.x)
        t[q] = keys[base + q];
    __syncthreads();
    for (int j = j0; j > 0; j >>= 1)
    {
        for (int q = threadIdx.x; q < kSortTile / 2; q += blockDim.x)
        {
            const int i = 2 * q - (q & (j - 1));
            const int64_t gi = base + i;
            cas(t[i], t[i + j], (gi & k) == 0);
        }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < kSortTile; q += blockDim.x)
        keys[base + q] = t[q];
}

// one stage at distance j >= kSortTile in global memory: one thread per pair
__global__ void k_bitonic_global(unsigned long long *__restrict__ keys, int64_t N, int64_t k, int64_t j)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N / 2)
        return;
    const int64_t i = 2 * q - (q & (j - 1));
    unsigned long long a = keys[i], b = keys[i + j];
    const bool up = (i & k) == 0;
    if ((a > b) == up)
    {
        keys[i] = b;
        keys[i + j] = a;
    }
}

cudaError_t bitonic_sort(cudaStream_t st, unsigned long long *keys, int64_t N)
{
    // N is a power of two >= kSortTile
    const int64_t tiles = N / kSortTile;
    k_bitonic_tile_full<<<(unsigned)tiles, kSortThreads, 0, st>>>(keys);
    for (int64_t k = 2 * kSortTile; k <= N; k <<= 1)
    {
        int64_t j = k >> 1;
        for (; j >= kSortTile; j >>= 1)
            k_bitonic_global<<<(unsigned)((N / 2 + 255) / 256), 256, 0, st>>>(keys, N, k, j);
        k_bitonic_tile_merge<<<(unsigned)tiles, kSortThreads, 0, st>>>(keys, k, (int)j);
    }
    return cudaGetLastError();
}

int64_t sort_size(int64_t n)
{
    int64_t N = kSortTile;
    while (N < n)
        N <<= 1;
    return N;
}

__global__ void k_pack_pairs(const int *__restrict__ key, int64_t n, int64_t N, unsigned long long *__restrict__ out)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N)
        return;
    out[q] = q < n ? ((unsigned long long)(unsigned)key[q] << 32) | (unsigned long long)(unsigned)q : ~0ull;
}

__global__ void k_unpack_pairs(const unsigned long long *__restrict__ s, int64_t n, const int *__restrict__ key,
                               const int *__restrict__ val, int *__restrict__ skey, int *__restrict__ sval)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n)
        return;
    const unsigned pos = (unsigned)(s[q] & 0xffffffffull);
    skey[q] = key[pos];
    sval[q] = val[pos];
}

// segment << 32 | value for every element; one warp per segment
__global__ void k_pack_segments(const int *__restrict__ in, int nseg, const int *__restrict__ off, int64_t total,
                                int64_t N, unsigned long long *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t sgi = w; sgi < nseg; sgi += nw)
        for (int64_t q = off[sgi] + lane; q < off[sgi + 1]; q += 32)
            out[q] = ((unsigned long long)sgi << 32) | (unsigned long long)(unsigned)in[q];
    for (int64_t q = total + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x); q < N;
         q += (int64_t)gridDim.x * blockDim.x)
        out[q] = ~0ull;
}

__global__ void k_unpack_segments(const unsigned long long *__restrict__ s, int64_t total, int *__restrict__ out)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < total)
        out[q] = (int)(unsigned)(s[q] & 0xffffffffull);
}

} // namespace

cudaError_t prim_exclusive_scan(cudaStream_t st, const int *in, int *out, int64_t count)
{
    return scan_impl<int>(st, in, out, count);
}

cudaError_t prim_exclusive_scan(cudaStream_t st, const int64_t *in, int64_t *out, int64_t count)
{
    return scan_impl<int64_t>(st, in, out, count);
}

cudaError_t prim_max(cudaStream_t st, const int *in, int64_t count, int *dev_out)
{
    k_max_one_block<<<1, 1024, 0, st>>>(in, count, dev_out);
    return cudaGetLastError();
}

cudaError_t prim_sort_pairs(cudaStream_t st, const int *key, const int *val, int *skey, int *sval, int64_t n)
{
    if (n <= 0)
        return cudaSuccess;
    const int64_t N = sort_size(n);
    unsigned long long *k64 = nullptr;
    cudaError_t e = cudaMallocAsync(&k64, sizeof(unsigned long long) * N, st);
    if (e != cudaSuccess)
        return e;
    k_pack_pairs<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(key, n, N, k64);
    if ((e = bitonic_sort(st, k64, N)) == cudaSuccess)
    {
        k_unpack_pairs<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(k64, n, key, val, skey, sval);
        e = cudaGetLastError();
    }
    cudaFreeAsync(k64, st);
    return e;
}

cudaError_t prim_segmented_sort(cudaStream_t st, const int *in, int *out, int64_t total, int nseg, const int *off)
{
    if (total <= 0)
        return cudaSuccess;
    const int64_t N = sort_size(total);
    unsigned long long *k64 = nullptr;
    cudaError_t e = cudaMallocAsync(&k64, sizeof(unsigned long long) * N, st);
    if (e != cudaSuccess)
        return e;
    k_pack_segments<<<1024, 256, 0, st>>>(in, nseg, off, total, N, k64);
    if ((e = bitonic_sort(st, k64, N)) == cudaSuccess)
    {
        k_unpack_segments<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(k64, total, out);
        e = cudaGetLastError();
    }
    cudaFreeAsync(k64, st);
    return e;
}

} // namespace lpm
