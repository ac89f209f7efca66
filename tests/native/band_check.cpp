// Test harness: runs the band Cholesky core of lpm-cpp_b200/csrc/band_chol.cuh on the host, in
// the order and with the thread decomposition the device driver (csrc/direct.cu: factor,
// substitute) uses, so the tests check the device's arithmetic on the CPU.
//
//   band_check IN OUT
// IN:  int64 n, int64 kd, int64 nb, then the lower band AB ((kd + 1) * n doubles, column j at
//      AB[j * (kd + 1)]) and the right-hand side b (n doubles)
// OUT: the solution x (n doubles), the factor (the band after factoring), int32 fail (0, or the
//      1-based column whose pivot was not positive)
#include <cstdint>
#include <cstdio>
#include <vector>

#include "band_chol.cuh"

using namespace lpm::band;

int main(int argc, char **argv)
{
    if (argc != 3)
        return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f)
        return 2;
    int64_t hdr[3];
    if (std::fread(hdr, sizeof(int64_t), 3, f) != 3)
        return 2;
    const int64_t n = hdr[0], kd = hdr[1], nb = hdr[2], ldab = kd + 1;
    std::vector<double> AB((size_t)(ldab * n)), y((size_t)n);
    if (std::fread(AB.data(), sizeof(double), AB.size(), f) != AB.size() ||
        std::fread(y.data(), sizeof(double), y.size(), f) != y.size())
        return 2;
    std::fclose(f);
    int fail = 0;
    // factor<D>: per column block, the diagonal block, the rows below, the trailing window
    for (int64_t j0 = 0; j0 < n; j0 += nb)
    {
        const int64_t jb = n - j0 < nb ? n - j0 : nb;
        const int64_t m2 = below_end(n, kd, j0, jb) - (j0 + jb);
        const int r = potrf_block(AB.data(), ldab, kd, j0, jb);
        if (r && fail == 0)
            fail = (int)(j0 + r);
        for (int64_t t = 0; t < m2; ++t)
            trsm_row(AB.data(), ldab, kd, j0, jb, j0 + jb + t);
        for (int64_t cy = 0; cy < m2; ++cy)
        {
            const int64_t c = j0 + jb + cy;
            for (int64_t i = c; i < j0 + jb + m2 && i - c <= kd; ++i)
                syrk_entry(AB.data(), ldab, kd, j0, jb, i, c);
        }
    }
    // substitute<D>: forward by blocks, then backward from the last block
    for (int64_t j0 = 0; j0 < n; j0 += nb)
    {
        const int64_t jb = n - j0 < nb ? n - j0 : nb;
        const int64_t m2 = below_end(n, kd, j0, jb) - (j0 + jb);
        fwd_block(AB.data(), ldab, kd, j0, jb, y.data());
        for (int64_t t = 0; t < m2; ++t)
            fwd_update_row(AB.data(), ldab, kd, j0, jb, j0 + jb + t, y.data());
    }
    for (int64_t j0 = ((n - 1) / nb) * nb; j0 >= 0; j0 -= nb)
    {
        const int64_t jb = n - j0 < nb ? n - j0 : nb;
        if (j0 + jb < n)
            for (int64_t t = 0; t < jb; ++t)
                bwd_update_col(AB.data(), ldab, kd, n, j0, jb, j0 + t, y.data());
        bwd_block(AB.data(), ldab, kd, j0, jb, y.data());
    }
    FILE *o = std::fopen(argv[2], "wb");
    if (!o)
        return 2;
    std::fwrite(y.data(), sizeof(double), y.size(), o);
    std::fwrite(AB.data(), sizeof(double), AB.size(), o);
    std::fwrite(&fail, sizeof(int), 1, o);
    std::fclose(o);
    return 0;
}
