// Host check of bph_direct.h: the closed-form eigenvectors of the vertical
// second difference are orthonormal and diagonalise it (E T E^T = diag
// lambda) for both bottom conditions and a range of heights.
#include <cmath>
#include <cstdio>
#include <vector>

#include "bph_direct.h"

int main() {
    int fails = 0;
    for (int isym : {1, 2})
        for (int nz : {1, 2, 3, 7, 16, 33, 96, 192}) {
            std::vector<long double> E, lam;
            bph::direct::vertical_eigen(nz, isym, E, lam);
            long double worst_o = 0.0L, worst_d = 0.0L;
            std::vector<long double> t(nz);
            for (int q = 0; q < nz; ++q) {
                bph::direct::apply_vertical(nz, isym, &E[(size_t)q * nz], t.data());
                for (int p = 0; p < nz; ++p) {
                    long double dot = 0.0L, td = 0.0L;
                    for (int k = 0; k < nz; ++k) {
                        dot += E[(size_t)p * nz + k] * E[(size_t)q * nz + k];
                        td += E[(size_t)p * nz + k] * t[k];
                    }
                    worst_o = std::fmax(worst_o, std::fabs(dot - (p == q ? 1.0L : 0.0L)));
                    worst_d = std::fmax(worst_d, std::fabs(td - (p == q ? lam[q] : 0.0L)));
                }
            }
            if (!(worst_o < 1e-15L && worst_d < 1e-15L)) {
                std::printf("isym %d nz %d: orthonormality %.3Le, diagonalisation %.3Le\n", isym, nz, worst_o, worst_d);
                ++fails;
            }
        }
    if (fails) {
        std::printf("%d checks failed\n", fails);
        return 1;
    }
    std::printf("all checks passed\n");
    return 0;
}
