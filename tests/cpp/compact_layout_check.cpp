// Host check of the compact Green-table layout (bph_compact.h) and of the
// index arithmetic of the contraction that reads it (k_green_compact):
// synthetic tables with the two symmetries of the Green function -- H
// symmetric in (jb, j) for the top and bottom rows, U(kb - k) + V(kb + k)
// for the side rows -- are packed in the compact layout, contracted the
// way the kernel does it (lane by lane: tile rows and columns, sliding side
// windows, the last CTA's sums over tiles and side CTAs), and compared with
// the dense contraction S[b] = sum_p G[b][p] mom[p].
#include <cmath>
#include <cstdio>
#include <vector>

#include "bph_compact.h"

using namespace bph::compact;

static int fails = 0;

static double h_sym(int set, int a, int b, int k) {
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    return 1.0 / (1.0 + 0.37 * lo + 0.11 * hi * hi + 0.05 * k) + 0.01 * set * std::cos(0.3 * (lo + hi) + k);
}
static double u_fn(int j, int d) { return std::exp(-0.05 * (d < 0 ? -d : d)) / (1.0 + j); }
static double v_fn(int j, int s) { return 0.3 * std::cos(0.1 * s + j) / (2.0 + j); }

static void check(int nr, int nz, int isym) {
    const Dims d = dims(nr, nz, isym);
    if (!d.ok) return;
    const bool image = isym != 1;
    const int nb = (isym == 1) ? 2 * nr + nz : nr + nz;
    const long long np = (long long)nr * nz;
    std::vector<double> rw(nr), mom(2 * np);
    for (int j = 0; j < nr; ++j) rw[j] = 0.5 + 0.1 * j;
    for (long long p = 0; p < 2 * np; ++p) mom[p] = std::sin(0.7 * p + 0.2) + 0.1;
    // dense reference
    std::vector<double> S_ref(2 * nb, 0.0);
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < nr; ++j) {
                double g;
                if (b < nr)
                    g = h_sym(0, b, j, k) * rw[j];
                else if (b < nr + nz)
                    g = u_fn(j, (b - nr) - k) + (image ? v_fn(j, (b - nr) + k) : 0.0);
                else
                    g = h_sym(1, b - nr - nz, j, k) * rw[j];
                S_ref[2 * b] += g * mom[j + (long long)nr * k];
                S_ref[2 * b + 1] += g * mom[np + j + (long long)nr * k];
            }
    // compact tables
    std::vector<double> T((size_t)pair_doubles(d), 0.0), Sd((size_t)side_doubles(d), 0.0);
    for (int set = 0; set < d.nsets; ++set)
        for (int q = 0; q < d.npair; ++q) {
            int I, J;
            pair_blocks(q, d.nb8, &I, &J);
            if (pair_index(I, J, d.nb8) != q || I > J) {
                std::printf("pair %d of %d: blocks (%d, %d) do not index back\n", q, d.nb8, I, J);
                ++fails;
            }
            for (int k = 0; k < nz; ++k)
                for (int e = 0; e < 64; ++e) {
                    const int jb = kTile * I + (e >> 3), j = kTile * J + (e & 7);
                    if (jb < nr && j < nr)
                        T[(((size_t)set * d.nzp + k) * d.npair + q) * 64 + e] = h_sym(set, jb, j, k);
                }
        }
    for (int j = 0; j < nr; ++j)
        for (int pos = 0; pos < d.stride; ++pos) {
            if (pos <= 2 * nz - 2) Sd[((size_t)j * 2) * d.stride + pos] = u_fn(j, pos - (nz - 1));
            if (image && pos <= 2 * nz - 2) Sd[((size_t)j * 2 + 1) * d.stride + pos] = v_fn(j, pos);
        }
    // the kernel's partial sums, per height part
    std::vector<double> part((size_t)part_doubles(d), 0.0);
    for (int h = 0; h < d.nh; ++h) {
    int k0, k1;
    height_range(d, h, &k0, &k1);
    double *parth = &part[(size_t)h * part_height_doubles(d)];
    for (int q = 0; q < d.nsets * d.npair; ++q) {
        const int set = q / d.npair, tile = q % d.npair;
        int I, J;
        pair_blocks(tile, d.nb8, &I, &J);
        double lane_r[32][2], lane_c[32][2][2];
        for (int lane = 0; lane < 32; ++lane) {
            const int r = lane >> 2, c0 = 2 * (lane & 3);
            const int jr = std::min(kTile * I + r, nr - 1);
            const int jc0 = std::min(kTile * J + c0, nr - 1), jc1 = std::min(kTile * J + c0 + 1, nr - 1);
            double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = k0; k < k1; ++k) {
                const double *t = &T[(((size_t)set * d.nzp + k) * d.npair + tile) * 64 + 2 * lane];
                const long long off = (long long)nr * k;
                const double xc0 = mom[off + jc0], xc1 = mom[off + jc1], xs0 = mom[np + off + jc0],
                             xs1 = mom[np + off + jc1], yc = mom[off + jr], ys = mom[np + off + jr];
                acc[0] += t[0] * xc0;
                acc[1] += t[0] * xs0;
                acc[2] += t[1] * xc1;
                acc[3] += t[1] * xs1;
                acc[4] += t[0] * yc;
                acc[5] += t[0] * ys;
                acc[6] += t[1] * yc;
                acc[7] += t[1] * ys;
            }
            lane_r[lane][0] = rw[jc0] * acc[0] + rw[jc1] * acc[2];
            lane_r[lane][1] = rw[jc0] * acc[1] + rw[jc1] * acc[3];
            lane_c[lane][0][0] = rw[jr] * acc[4];
            lane_c[lane][0][1] = rw[jr] * acc[5];
            lane_c[lane][1][0] = rw[jr] * acc[6];
            lane_c[lane][1][1] = rw[jr] * acc[7];
        }
        double *pp = &parth[(size_t)q * kPartPair];
        for (int r = 0; r < 8; ++r)
            for (int cs = 0; cs < 2; ++cs) {
                double v = 0.0;
                for (int x = 0; x < 4; ++x) v += lane_r[4 * r + x][cs];
                pp[2 * r + cs] = v;
            }
        for (int x = 0; x < 4; ++x)
            for (int h = 0; h < 2; ++h)
                for (int cs = 0; cs < 2; ++cs) {
                    double v = 0.0;
                    for (int r = 0; r < 8; ++r) v += lane_c[4 * r + x][h][cs];
                    pp[16 + 2 * (2 * x + h) + cs] = v;
                }
    }
    for (int g = 0; g < d.side_ctas; ++g) {
        std::vector<double> cta(2 * 32 * d.kpl, 0.0);
        for (int w = 0; w < kWarps; ++w) {
            const int j = g * kWarps + w;
            if (j >= nr) continue;
            const double *Uv = &Sd[(size_t)j * 2 * d.stride], *Vv = Uv + d.stride;
            for (int lane = 0; lane < 32; ++lane) {
                const int base = d.kpl * lane;
                const int K = d.kpl;
                double uu[kMaxKpl], vv[kMaxKpl], ac[kMaxKpl] = {0}, as[kMaxKpl] = {0};
                for (int i = 0; i < K; ++i) {
                    uu[i] = Uv[base + i + nz - 1 - k0];
                    vv[i] = Vv[base + i + k0];
                }
                for (int kb = k0; kb < k1; kb += K)
                    for (int st = 0; st < K; ++st) {
                        const int k = kb + st;
                        if (k >= k1) continue;
                        const double xc = mom[j + (long long)nr * k], xs = mom[np + j + (long long)nr * k];
                        const int vi = base + K + k;
                        if (vi >= d.stride) {
                            std::printf("nr %d nz %d: V window index %d past stride %d\n", nr, nz, vi, d.stride);
                            ++fails;
                            return;
                        }
                        const double un = (k + 1 < k1) ? Uv[base + nz - 2 - k] : 0.0;
                        const double vn = (k + 1 < k1) ? Vv[vi] : 0.0;
                        for (int i = 0; i < K; ++i) {
                            const double ww = uu[(i - st + K) % K] + vv[(i + st) % K];
                            ac[i] += ww * xc;
                            as[i] += ww * xs;
                        }
                        uu[K - 1 - st] = un;
                        vv[st] = vn;
                    }
                for (int i = 0; i < d.kpl; ++i) {
                    cta[2 * (base + i)] += ac[i];
                    cta[2 * (base + i) + 1] += as[i];
                }
            }
        }
        double *ps = &parth[(size_t)d.nsets * d.npair * kPartPair + (size_t)g * nz * 2];
        for (int kb = 0; kb < nz; ++kb) {
            ps[2 * kb] = cta[2 * kb];
            ps[2 * kb + 1] = cta[2 * kb + 1];
        }
    }
    }
    // level 2: each tile set's / side group's height parts added; level 3: per boundary row
    const size_t ph = (size_t)part_height_doubles(d);
    std::vector<double> merged(ph, 0.0);
    for (size_t e = 0; e < ph; ++e)
        for (int h = 0; h < d.nh; ++h) merged[e] += part[(size_t)h * ph + e];
    double worst = 0.0, scale = 0.0;
    for (int b = 0; b < nb; ++b) {
        double sc = 0.0, ss = 0.0;
        if (b < nr || b >= nr + nz) {
            const int set = (b < nr) ? 0 : 1;
            const int jb = (b < nr) ? b : b - nr - nz;
            const int I = jb / kTile, r = jb % kTile;
            const double *pt = &merged[(size_t)set * d.npair * kPartPair];
            for (int t = 0; t < d.nb8; ++t) {
                const double *pp = (t < I) ? pt + (size_t)pair_index(t, I, d.nb8) * kPartPair + 16 + 2 * r
                                           : pt + (size_t)pair_index(I, t, d.nb8) * kPartPair + 2 * r;
                sc += pp[0];
                ss += pp[1];
            }
        } else {
            const double *pside = &merged[(size_t)d.nsets * d.npair * kPartPair];
            for (int g = 0; g < d.side_ctas; ++g) {
                sc += pside[((size_t)g * nz + (b - nr)) * 2];
                ss += pside[((size_t)g * nz + (b - nr)) * 2 + 1];
            }
        }
        worst = std::fmax(worst, std::fmax(std::fabs(sc - S_ref[2 * b]), std::fabs(ss - S_ref[2 * b + 1])));
        scale = std::fmax(scale, std::fmax(std::fabs(S_ref[2 * b]), std::fabs(S_ref[2 * b + 1])));
    }
    if (!(worst <= 1e-12 * scale)) {
        std::printf("nr %d nz %d isym %d: compact contraction differs by %.3e (scale %.3e)\n", nr, nz, isym, worst,
                    scale);
        ++fails;
    }
}

int main() {
    const int nrs[] = {3, 8, 13, 16, 33, 64};
    const int nzs[] = {1, 2, 3, 5, 7, 32, 33, 70, 96};
    for (int nr : nrs)
        for (int nz : nzs)
            for (int isym : {1, 2}) check(nr, nz, isym);
    // parts and tiles of the production grid 130 x 98
    const Dims d = dims(128, 96, 2);
    if (d.npair != 136 || d.kpl != 3 || d.top_ctas != 17 || d.side_ctas != 16 || d.nh != 1 || d.hp != 96 || d.nzp != 96 ||
        items(d, 30) != 30 * 33) {
        std::printf("130 x 98 dims: npair %d kpl %d top %d side %d nh %d hp %d\n", d.npair, d.kpl, d.top_ctas,
                    d.side_ctas, d.nh, d.hp);
        ++fails;
    }
    if (dims(128, 257, 2).ok) {
        std::printf("nz 257 should fall back to the full tables\n");
        ++fails;
    }
    if (fails) {
        std::printf("%d checks failed\n", fails);
        return 1;
    }
    std::printf("all checks passed\n");
    return 0;
}
