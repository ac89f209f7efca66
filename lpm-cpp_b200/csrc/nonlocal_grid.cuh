// Cell-grid candidates of the nonlocal neighbour search (Assembly::searchNonlocalNeighbors,
// include/assembly.h:118-130): the particles j within distance rc of particle i, found among the
// particles of i's cell and the cells around it.  Cells are at least rc wide (with a margin for
// the rounding of the binning), so every j with distanceTo < rc lies in a neighbouring cell.
// The distance is Particle::distanceTo (particle.h:277-280) with pow(x, 2) as x * x, as in the
// all-pairs search, so the neighbour sets are the same; the caller sorts each list into the
// reference's order (ascending id).  One call is the whole work of one thread; it compiles as
// device and host code, and the tests run it on the CPU.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define LPM_HD_NL __host__ __device__ __forceinline__
#else
#define LPM_HD_NL inline
#endif

namespace lpm
{
namespace nlgrid
{

LPM_HD_NL double distance(const double *xyz, int i, int j)
{
    const double dx = xyz[3 * i] - xyz[3 * j], dy = xyz[3 * i + 1] - xyz[3 * j + 1], dz = xyz[3 * i + 2] - xyz[3 * j + 2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// cell (cx, cy, cz) -> linear index, x fastest
LPM_HD_NL int64_t cell_index(int cx, int cy, int cz, const int *dims)
{
    return ((int64_t)cz * dims[1] + cy) * dims[0] + cx;
}

// The j (any order) with distance(i, j) < rc among the cells around i's cell (cxyz: i's cell
// coordinates); cell c holds cell_ids[cell_start[c] .. cell_start[c + 1]).  Writes them to out
// when out != nullptr; returns their count.
LPM_HD_NL int candidates(int i, const double *xyz, double rc, const int *cxyz, const int *dims,
                         const int *cell_start, const int *cell_ids, int *out)
{
    int c = 0;
    for (int dz = -1; dz <= 1; ++dz)
    {
        const int z = cxyz[2] + dz;
        if (z < 0 || z >= dims[2])
            continue;
        for (int dy = -1; dy <= 1; ++dy)
        {
            const int y = cxyz[1] + dy;
            if (y < 0 || y >= dims[1])
                continue;
            for (int dx = -1; dx <= 1; ++dx)
            {
                const int x = cxyz[0] + dx;
                if (x < 0 || x >= dims[0])
                    continue;
                const int64_t cell = cell_index(x, y, z, dims);
                for (int k = cell_start[cell]; k < cell_start[cell + 1]; ++k)
                {
                    const int j = cell_ids[k];
                    if (distance(xyz, i, j) < rc)
                    {
                        if (out)
                            out[c] = j;
                        ++c;
                    }
                }
            }
        }
    }
    return c;
}

// Host binning (host code only): cells of side h >= rc (1e-9 wider, so that rounding in the binning never puts two
// particles closer than rc two cells apart), widened further while the grid would exceed
// max_cells.  cxyz[3 i ..] gets particle i's cell; cell_start / cell_ids list each cell's
// particles in ascending id.  Returns false for rc <= 0 or no particles.
template <typename IntVec>
inline bool bin(const double *xyz, int n, double rc, int64_t max_cells, int dims[3], IntVec &cxyz,
                IntVec &cell_start, IntVec &cell_ids)
{
    if (!(rc > 0) || n <= 0)
        return false;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a)
    {
        lo[a] = hi[a] = xyz[a];
        for (int i = 1; i < n; ++i)
        {
            lo[a] = xyz[3 * i + a] < lo[a] ? xyz[3 * i + a] : lo[a];
            hi[a] = xyz[3 * i + a] > hi[a] ? xyz[3 * i + a] : hi[a];
        }
    }
    double h = rc * (1.0 + 1e-9);
    for (;;)
    {
        int64_t total = 1;
        for (int a = 0; a < 3; ++a)
        {
            dims[a] = (int)std::floor((hi[a] - lo[a]) / h) + 1;
            total *= dims[a];
        }
        if (total <= max_cells)
            break;
        h *= 2.0;
    }
    cxyz.assign((size_t)3 * n, 0);
    const int64_t ncell = (int64_t)dims[0] * dims[1] * dims[2];
    cell_start.assign((size_t)ncell + 1, 0);
    for (int i = 0; i < n; ++i)
    {
        for (int a = 0; a < 3; ++a)
        {
            int c = (int)std::floor((xyz[3 * i + a] - lo[a]) / h);
            c = c < 0 ? 0 : (c >= dims[a] ? dims[a] - 1 : c);
            cxyz[3 * i + a] = c;
        }
        cell_start[cell_index(cxyz[3 * i], cxyz[3 * i + 1], cxyz[3 * i + 2], dims) + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c)
        cell_start[c + 1] += cell_start[c];
    cell_ids.assign((size_t)n, 0);
    IntVec fill(cell_start.begin(), cell_start.end() - 1);
    for (int i = 0; i < n; ++i)
        cell_ids[fill[cell_index(cxyz[3 * i], cxyz[3 * i + 1], cxyz[3 * i + 2], dims)]++] = i;
    return true;
}

} // namespace nlgrid
} // namespace lpm
