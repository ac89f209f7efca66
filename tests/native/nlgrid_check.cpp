// Test harness: the cell-grid nonlocal search of lpm-cpp_b200/csrc/nonlocal_grid.cuh on the host
// (the binning, and the per-particle candidates the device kernel collects, each list then sorted
// as the device's segmented sort sorts it), against the all-pairs search in the reference's loop
// order (assembly.h:118-130).
//
//   nlgrid_check IN MAX_CELLS      IN: int64 n, double rc, then xyz (3 n doubles)
// prints "<particles whose lists differ> <total pairs>"
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "nonlocal_grid.cuh"

int main(int argc, char **argv)
{
    if (argc != 3)
        return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f)
        return 2;
    int64_t n64;
    double rc;
    if (std::fread(&n64, sizeof n64, 1, f) != 1 || std::fread(&rc, sizeof rc, 1, f) != 1)
        return 2;
    const int n = (int)n64;
    std::vector<double> xyz((size_t)3 * n);
    if (std::fread(xyz.data(), sizeof(double), xyz.size(), f) != xyz.size())
        return 2;
    std::fclose(f);
    int dims[3];
    std::vector<int> cxyz, cell_start, cell_ids;
    if (!lpm::nlgrid::bin(xyz.data(), n, rc, std::atoll(argv[2]), dims, cxyz, cell_start, cell_ids))
        return 3;
    int bad = 0;
    int64_t pairs = 0;
    std::vector<int> got, want;
    for (int i = 0; i < n; ++i)
    {
        const int c = lpm::nlgrid::candidates(i, xyz.data(), rc, cxyz.data() + 3 * i, dims, cell_start.data(),
                                              cell_ids.data(), nullptr);
        got.assign(c, -1);
        lpm::nlgrid::candidates(i, xyz.data(), rc, cxyz.data() + 3 * i, dims, cell_start.data(), cell_ids.data(),
                                got.data());
        std::sort(got.begin(), got.end());
        want.clear();
        for (int j = 0; j < n; ++j)
            if (lpm::nlgrid::distance(xyz.data(), i, j) < rc)
                want.push_back(j);
        bad += got != want;
        pairs += c;
    }
    std::printf("%d %lld\n", bad, (long long)pairs);
    return 0;
}
