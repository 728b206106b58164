// Index arithmetic of the direct defect-solve kernel (bph_direct.h), run on
// the CPU with the kernel's schedule emulated lane by lane:
//  * the fragment offsets address the elements that the m16n8k8 TF32
//    fragment layout assigns to each lane (A row-major, B column-major,
//    D row-major, PTX ISA "Matrix fragments for mma.m16n8k8");
//  * the in-place transform (products of a block formed, then written) over
//    the warp tiles equals the dense product E X, every output written once,
//    every access inside the shared-memory arrays;
//  * the residual sweep (a warp per 32 columns and band of rows, neighbours
//    by shuffle) gives the per-zone FP64 residual bit for bit and reads only
//    inside the slot arrays;
//  * the twisted factorization of the radial systems (two sides, meeting
//    rows, back substitution) solves them to FP32 accuracy for odd, even
//    and single-row lengths.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "bph_direct.h"

using namespace bph::direct;

static int failures = 0;
#define CHECK(c, ...)                      \
    do {                                   \
        if (!(c)) {                        \
            ++failures;                    \
            if (failures < 20) {           \
                std::printf("FAIL: ");     \
                std::printf(__VA_ARGS__);  \
                std::printf("\n");         \
            }                              \
        }                                  \
    } while (0)

// Documented lane layout of mma.m16n8k8 (tf32): (row, column) of value v.
static void a_elem(int g, int t, int v, int &r, int &c) {
    r = g + ((v == 1 || v == 3) ? 8 : 0);
    c = t + ((v >= 2) ? 4 : 0);
}
static void b_elem(int g, int t, int v, int &k, int &n) {
    k = t + (v ? 4 : 0);
    n = g;
}
static void d_elem(int g, int t, int v, int &r, int &c) {
    r = g + ((v >= 2) ? 8 : 0);
    c = 2 * t + (v & 1);
}

static void check_fragments() {
    const int lda = 100, ldk = 132;
    for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, t = lane & 3;
        for (int m = 0; m < 2; ++m)
            for (int v = 0; v < 4; ++v) {
                int r, c;
                a_elem(g, t, v, r, c);
                CHECK(a_offset(32, m, 8, g, t, lda, v) == (32 + 16 * m + r) * lda + 8 + c, "a lane %d v %d", lane, v);
                d_elem(g, t, v, r, c);
                // the result element (mode row, column j) is stored transposed: X^T[j][mode]
                for (int n = 0; n < 2; ++n)
                    CHECK(d_offset(32, m, 16, n, g, t, ldk, v) == (16 + 8 * n + c) * ldk + 32 + 16 * m + r,
                          "d lane %d v %d", lane, v);
            }
        for (int n = 0; n < 2; ++n)
            for (int v = 0; v < 2; ++v) {
                int k, col;
                b_elem(g, t, v, k, col);
                CHECK(b_offset(16, n, 8, g, t, ldk, v) == (16 + 8 * n + col) * ldk + 8 + k, "b lane %d v %d", lane, v);
            }
    }
}

// X <- A X on X^T [nrp][ldk] with the kernel's blocks and warp tiles.
static void emulate_transform(const Shape &d, const std::vector<double> &A, std::vector<double> &Xt,
                              std::vector<int> &writes) {
    const int cp = d.nrp / 16;
    for (int cp0 = 0; cp0 < cp; cp0 += d.cpb) {
        const int ncp = (d.cpb < cp - cp0) ? d.cpb : cp - cp0, tiles = (d.nzp / 32) * ncp;
        CHECK(tiles <= kBlockTiles, "block of %d tiles", tiles);
        struct Out {
            int off;
            double val;
        };
        std::vector<Out> outs;
        for (int w = 0; w < kWarps; ++w)
            for (int r = 0; r < kTilesPerWarp; ++r) {
                const int tile = w + kWarps * r;
                if (tile >= tiles) continue;
                int i0, c0;
                warp_tile(tile, cp0, ncp, i0, c0);
                for (int m = 0; m < 2; ++m)
                    for (int n = 0; n < 2; ++n) {
                        double acc[32][4] = {};
                        for (int k0 = 0; k0 < d.nzp; k0 += 8) {
                            double At[16][8], Bt[8][8];  // the sub-tile operands gathered from the lanes
                            for (int lane = 0; lane < 32; ++lane) {
                                const int g = lane >> 2, t = lane & 3;
                                for (int v = 0; v < 4; ++v) {
                                    const int o = a_offset(i0, m, k0, g, t, d.lda, v);
                                    CHECK(o >= 0 && o < d.nzp * d.lda, "A offset %d", o);
                                    int rr, cc;
                                    a_elem(g, t, v, rr, cc);
                                    At[rr][cc] = A[o];
                                }
                                for (int v = 0; v < 2; ++v) {
                                    const int o = b_offset(c0, n, k0, g, t, d.ldk, v);
                                    CHECK(o >= 0 && o < d.nrp * d.ldk && o % d.ldk < d.nzp, "B offset %d", o);
                                    int kk, nn;
                                    b_elem(g, t, v, kk, nn);
                                    Bt[kk][nn] = Xt[o];
                                }
                            }
                            for (int lane = 0; lane < 32; ++lane) {
                                const int g = lane >> 2, t = lane & 3;
                                for (int v = 0; v < 4; ++v) {
                                    int rr, cc;
                                    d_elem(g, t, v, rr, cc);
                                    for (int k = 0; k < 8; ++k) acc[lane][v] += At[rr][k] * Bt[k][cc];
                                }
                            }
                        }
                        for (int lane = 0; lane < 32; ++lane)
                            for (int v = 0; v < 4; ++v) {
                                const int o = d_offset(i0, m, c0, n, lane >> 2, lane & 3, d.ldk, v);
                                CHECK(o >= 0 && o < d.nrp * d.ldk && o % d.ldk < d.nzp, "D offset %d", o);
                                // a write may only land on columns j of this block
                                const int j = o / d.ldk;
                                CHECK(j >= 16 * cp0 && j < 16 * (cp0 + ncp), "write outside the block");
                                outs.push_back({o, acc[lane][v]});
                            }
                    }
            }
        for (const Out &o : outs) {  // after the block's barrier
            Xt[o.off] = o.val;
            ++writes[o.off];
        }
    }
}

static void check_transform(int nr, int nz, std::mt19937 &rng) {
    const Shape d = shape(nr, nz);
    if (d.cpb == 0) return;
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<double> A((size_t)d.nzp * d.lda, 0.0), X((size_t)nz * nr), Xt((size_t)d.nrp * d.ldk, 0.0);
    for (int q = 0; q < nz; ++q)
        for (int k = 0; k < nz; ++k) A[(size_t)q * d.lda + k] = u(rng);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < nr; ++j) {
            X[(size_t)k * nr + j] = u(rng);
            Xt[(size_t)j * d.ldk + k] = X[(size_t)k * nr + j];
        }
    std::vector<int> writes(Xt.size(), 0);
    emulate_transform(d, A, Xt, writes);
    double err = 0.0;
    for (int j = 0; j < d.nrp; ++j)
        for (int q = 0; q < d.nzp; ++q) {
            CHECK(writes[(size_t)j * d.ldk + q] == 1, "nr %d nz %d: (%d, %d) written %d times", nr, nz, q, j,
                  writes[(size_t)j * d.ldk + q]);
            double ref = 0.0;
            if (q < nz && j < nr)
                for (int k = 0; k < nz; ++k) ref += A[(size_t)q * d.lda + k] * X[(size_t)k * nr + j];
            err = std::fmax(err, std::fabs(Xt[(size_t)j * d.ldk + q] - ref));
        }
    CHECK(err < 1e-12, "nr %d nz %d: transform error %g", nr, nz, err);
    std::printf("nr %3d nz %3d: cpb %d, %zu bytes of shared memory, max error %.2e\n", nr, nz, d.cpb,
                d.floats * sizeof(float), err);
}

// The residual r = R - A phi: per zone (the reference statement) and by the
// kernel's sweep, both in FP64 with the same operation order.
static void check_residual(int nr, int nz, int isym, std::mt19937 &rng) {
    const int numr = nr + 2, numz = nz + 2;
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<double> P((size_t)numr * numz), R((size_t)nr * nz), brb(numr), alphar(numr), betar(numr), bzb(numz);
    for (auto &x : P) x = u(rng);
    for (auto &x : R) x = u(rng);
    for (auto &x : brb) x = u(rng);
    for (auto &x : alphar) x = u(rng);
    for (auto &x : betar) x = u(rng);
    for (auto &x : bzb) x = u(rng);
    const double gamma = 0.37;
    std::vector<double> ref((size_t)nr * nz), got((size_t)nr * nz, NAN);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < nr; ++j) {
            const double *pc = &P[(size_t)numr * (k + 1) + 1 + j];
            const double c = pc[0], ea = pc[1], no = pc[numr];
            const double we = (j > 0) ? pc[-1] : 0.0;
            const double so = (k > 0 || isym == 1) ? pc[-numr] : 0.0;
            const double ar = brb[j + 1] * c + alphar[j + 1] * ea + betar[j + 1] * we;
            const double az = bzb[k + 1] * c - gamma * no - gamma * so;
            ref[(size_t)k * nr + j] = R[(size_t)k * nr + j] - ar - az;
        }
    auto at = [&](long long off) {
        CHECK(off >= 0 && off < (long long)P.size(), "P read %lld outside the slot", off);
        return (off >= 0 && off < (long long)P.size()) ? P[(size_t)off] : 0.0;
    };
    for (int it = 0; it < sweep_items(nr); ++it) {
        int jc, k0, k1;
        sweep_item(it, nr, nz, jc, k0, k1);
        if (k0 >= k1) continue;
        double so[32], c[32];
        for (int lane = 0; lane < 32; ++lane) {
            const int j = jc + lane;
            const long long col = ((j < nr) ? j : nr) + 1;
            so[lane] = (k0 > 0 || isym == 1) ? at(col + (long long)numr * k0) : 0.0;
            c[lane] = at(col + (long long)numr * (k0 + 1));
        }
        for (int k = k0; k < k1; ++k) {
            double no[32], val[32];
            for (int lane = 0; lane < 32; ++lane) {
                const int j = jc + lane;
                const bool on = j < nr;
                const long long col = ((j < nr) ? j : nr) + 1;
                no[lane] = at(col + (long long)numr * (k + 2));
                double ea = c[(lane + 1) & 31];  // shfl_down by 1 (lane 31 keeps its own, replaced below)
                double we = c[(lane + 31) & 31];
                if (lane == 31) ea = c[31];
                if (lane == 0) we = c[0];
                if (lane == 31 && on) ea = at(col + (long long)numr * (k + 1) + 1);
                if (lane == 0) we = (j > 0) ? at(col + (long long)numr * (k + 1) - 1) : 0.0;
                const double br = on ? brb[j + 1] : 0.0, al = on ? alphar[j + 1] : 0.0, be = on ? betar[j + 1] : 0.0;
                const double rr = on ? R[(size_t)k * nr + j] : 0.0;
                const double ar = br * c[lane] + al * ea + be * we;
                const double az = bzb[k + 1] * c[lane] - gamma * no[lane] - gamma * so[lane];
                val[lane] = rr - ar - az;
                if (on) {
                    CHECK(std::isnan(got[(size_t)k * nr + j]), "zone (%d, %d) swept twice", k, j);
                    got[(size_t)k * nr + j] = val[lane];
                }
            }
            for (int lane = 0; lane < 32; ++lane) {
                so[lane] = c[lane];
                c[lane] = no[lane];
            }
        }
    }
    for (size_t e = 0; e < ref.size(); ++e)
        CHECK(got[e] == ref[e], "nr %d nz %d isym %d: zone %zu %.17g vs %.17g", nr, nz, isym, e, got[e], ref[e]);
}

// The twisted factorization of the kernel (both sides' elimination, the
// barrier, meeting, substitution, meeting rows) against an FP64 Thomas
// solve of the same diagonally dominant system; strided storage as in
// shared memory.
static void check_twisted(int n, std::mt19937 &rng) {
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const int ys = 5, cs = 3;
    std::vector<double> b(n);
    std::vector<float> lo(n), up(n), y((size_t)n * ys, NAN), c((size_t)n * cs, NAN);
    std::vector<double> v(n);
    for (int j = 0; j < n; ++j) {
        b[j] = 4.0 + u(rng);
        lo[j] = (float)u(rng);
        up[j] = (float)u(rng);
        v[j] = u(rng);
        y[(size_t)j * ys] = (float)v[j];
    }
    const double sigma = 0.37;
    Radial t;
    t.b = b.data();
    t.lo = lo.data();
    t.up = up.data();
    t.sigma = sigma;
    t.n = n;
    for (int side = 0; side < 2; ++side) twisted_eliminate<8>(t, side, y.data(), ys, c.data(), cs);
    float x0, x1;
    for (int side = 0; side < 2; ++side) {
        twisted_meet(t, y.data(), ys, c.data(), cs, x0, x1);
        twisted_substitute<8>(t, side, side ? x1 : x0, y.data(), ys, c.data(), cs);
    }
    twisted_meet(t, y.data(), ys, c.data(), cs, x0, x1);
    if (n / 2 > 0) y[(size_t)(n / 2 - 1) * ys] = x0;
    y[(size_t)(n / 2) * ys] = x1;
    // FP64 Thomas with the boundary couplings (lo_0, up_{n-1}) left out
    std::vector<double> cp(n), dp(n), x(n);
    for (int j = 0; j < n; ++j) {
        const double l = (j > 0) ? lo[j] : 0.0, m = b[j] + sigma - l * (j > 0 ? cp[j - 1] : 0.0);
        cp[j] = (j + 1 < n) ? up[j] / m : 0.0;
        dp[j] = (v[j] - l * (j > 0 ? dp[j - 1] : 0.0)) / m;
    }
    for (int j = n - 1; j >= 0; --j) x[j] = dp[j] - ((j + 1 < n) ? cp[j] * x[j + 1] : 0.0);
    double err = 0.0, nx = 0.0;
    for (int j = 0; j < n; ++j) {
        err = std::fmax(err, std::fabs((double)y[(size_t)j * ys] - x[j]));
        nx = std::fmax(nx, std::fabs(x[j]));
    }
    CHECK(err <= 1e-5 * nx, "twisted solve n %d: error %g of %g", n, err, nx);
}

int main() {
    check_fragments();
    std::mt19937 rng(7);
    const int shapes[][2] = {{128, 96}, {30, 14}, {62, 46}, {17, 33}, {8, 8}, {250, 60}, {128, 200}, {40, 100}};
    for (const auto &s : shapes) {
        check_transform(s[0], s[1], rng);
        for (int isym = 1; isym <= 3; ++isym) check_residual(s[0], s[1], isym, rng);
    }
    for (int n : {1, 2, 3, 4, 8, 9, 17, 37, 128, 250}) check_twisted(n, rng);
    const Shape p = shape(128, 96);
    CHECK(p.cpb == 8 && p.nzp == 96 && p.nrp == 128, "production shape cpb %d", p.cpb);
    CHECK(2 * (p.floats * sizeof(float) + 128 + 1024) <= 228u * 1024u, "two CTAs per SM: %zu bytes", p.floats * 4);
    for (const auto &s : shapes) {  // the regions: aligned, and the Thomas ratios fit the transform's region
        const Shape d = shape(s[0], s[1]);
        CHECK(d.off_bd % 2 == 0 && d.off_ms % 4 == 0, "nr %d nz %d: region alignment", s[0], s[1]);
        CHECK(d.off_lo - d.off_ms >= (size_t)d.nzp * d.lda && d.off_lo - d.off_ms >= (size_t)s[0] * s[1],
              "nr %d nz %d: transform region", s[0], s[1]);
        CHECK(d.off_ms - d.off_bd >= 2 * (size_t)s[0] && d.floats - d.off_up == (size_t)s[0], "nr %d nz %d: coefficients",
              s[0], s[1]);
    }
    CHECK(shape(30, 800).cpb == 0, "a slot of 800 modes is not offered");
    if (failures) {
        std::printf("%d failures\n", failures);
        return 1;
    }
    std::printf("all checks passed\n");
    return 0;
}
