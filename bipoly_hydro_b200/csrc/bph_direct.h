// bph_direct.h -- eigen-decomposition of the vertical ADI operator, for the
// direct defect solve of the mixed-precision converged forms.
//
// After the azimuthal transform every Fourier slot is a 2-D (r, z) system
// A = A_r (x) I + I (x) A_z: A_r is the radial tridiagonal of the slot
// (diagonal brb, off-diagonals alphar / betar, helmadi.F90:195-260) and
// A_z = gamma T with T the constant vertical second difference
// (bzb = 2 gamma, and gamma in the first row when the equatorial plane
// reflects: helmadi.F90:285-340), Dirichlet at the top.  T is diagonalised
// in closed form:
//   reflecting bottom (isym 2, 3): v_q(k) = cos((k + 1/2) theta_q),
//                                   theta_q = (q + 1/2) pi / (nz + 1/2);
//   Dirichlet bottom (isym 1):      v_q(k) = sin((k + 1) theta_q),
//                                   theta_q = (q + 1) pi / (nz + 1);
//   eigenvalue lambda_q = 2 - 2 cos theta_q.
// With E the orthonormal eigenvector matrix (rows q), A x = r becomes
// (A_r + gamma lambda_q) y_q = (E r)_q for every vertical mode q, and
// x = E^T y: one transform, nz radial tridiagonal solves, one transform.
// Plain C++ (long double), shared by the set-up and a host-side check,
// with the index arithmetic of the solve kernel (host and device).
#pragma once

#include <cmath>
#include <cstddef>
#include <vector>

#if defined(__CUDACC__)
#define BPH_DIRECT_HD __host__ __device__ __forceinline__
#define BPH_DIRECT_UNROLL _Pragma("unroll")
#else
#define BPH_DIRECT_HD inline
#define BPH_DIRECT_UNROLL
#endif

namespace bph {
namespace direct {

constexpr int kThreads = 256;                      // one CTA per (block row, slot), two per SM
constexpr int kWarps = kThreads / 32;
constexpr int kTilesPerWarp = 3;                   // 32 x 16 warp tiles per warp and transform block
constexpr int kBlockTiles = kTilesPerWarp * kWarps;  // 24: a 96 x 128 slot in one block

// Shared-memory shape of a slot of nr x nz interior zones, in floats from
// the start: X^T [nrp][ldk] (row j = column j of the [k][j] slot matrix);
// the radial diagonal of the slot [nr] (FP64, at off_bd); the transform
// [nzp][lda], which holds the Thomas ratios c' [nr][nz] between the two
// transforms (at off_ms); the radial sub- and super-diagonals [nr] (float,
// at off_lo and off_up).  Both strides are 4 modulo the 32 banks.
// cpb = column pairs (16 columns) per transform block; 0 when one block
// row of 32 modes already needs more warp tiles than the CTA holds.
struct Shape {
    int nrp, nzp, ldk, lda, cpb;
    size_t off_bd, off_ms, off_lo, off_up, floats;
};
BPH_DIRECT_HD Shape shape(int nr, int nz) {
    Shape d;
    d.nrp = (nr + 15) / 16 * 16;
    d.nzp = (nz + 31) / 32 * 32;
    d.ldk = d.nzp + 4;
    d.lda = d.nzp + 4;
    const int rp = d.nzp / 32, cp = d.nrp / 16;
    d.cpb = (rp > kBlockTiles) ? 0 : ((cp < kBlockTiles / rp) ? cp : kBlockTiles / rp);
    const size_t ms = (size_t)d.nzp * d.lda, cr = (size_t)nr * nz;
    d.off_bd = (size_t)d.nrp * d.ldk;                     // a multiple of 64 floats
    d.off_ms = d.off_bd + 2 * (((size_t)nr + 1) / 2 * 2);  // 16-byte aligned for the vector copies
    d.off_lo = d.off_ms + ((ms > cr ? ms : cr) + 3) / 4 * 4;
    d.off_up = d.off_lo + (size_t)nr;
    d.floats = d.off_up + (size_t)nr;
    return d;
}

// Warp tile `tile` of the transform block starting at column pair cp0 with
// ncp column pairs: its first output row (mode) i0 and column c0.
BPH_DIRECT_HD void warp_tile(int tile, int cp0, int ncp, int &i0, int &c0) {
    i0 = 32 * (tile / ncp);
    c0 = 16 * (cp0 + tile % ncp);
}
// m16n8k8 fragments of lane (g = lane / 4, t = lane % 4) in the warp tile
// (i0, c0), sub-tile (m, n), k-step k0, as word offsets:
//   A [nzp][lda]: a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4);
//   X^T [nrp][ldk]: b0 (k = t, n = g), b1 (k = t + 4, n = g);
//   X^T for the result: d0 (g, 2t), d1 (g, 2t + 1), d2 (g + 8, 2t),
//   d3 (g + 8, 2t + 1) of the 16 x 8 sub-tile, row = mode, column = j.
BPH_DIRECT_HD int a_offset(int i0, int m, int k0, int g, int t, int lda, int v) {
    return (i0 + 16 * m + g + 8 * (v & 1)) * lda + k0 + t + 4 * (v >> 1);
}
BPH_DIRECT_HD int b_offset(int c0, int n, int k0, int g, int t, int ldk, int v) {
    return (c0 + 8 * n + g) * ldk + k0 + t + 4 * v;
}
BPH_DIRECT_HD int d_offset(int i0, int m, int c0, int n, int g, int t, int ldk, int v) {
    return (c0 + 8 * n + 2 * t + (v & 1)) * ldk + i0 + 16 * m + g + 8 * (v >> 1);
}

// Residual sweep item `it` of kWarps warps: columns jc .. jc + 31 and rows
// [k0, k1) (k0 >= k1: nothing); items = column chunks x bands.
BPH_DIRECT_HD int sweep_items(int nr) {
    const int nchunk = (nr + 31) / 32;
    return nchunk * ((kWarps / nchunk > 1) ? kWarps / nchunk : 1);
}
BPH_DIRECT_HD void sweep_item(int it, int nr, int nz, int &jc, int &k0, int &k1) {
    const int nchunk = (nr + 31) / 32;
    const int nband = (kWarps / nchunk > 1) ? kWarps / nchunk : 1;
    const int band_rows = (nz + nband - 1) / nband;
    jc = (it % nchunk) * 32;
    k0 = (it / nchunk) * band_rows;
    k1 = (k0 + band_rows < nz) ? k0 + band_rows : nz;
}

// E (nz x nz, row q = eigenvector q, orthonormal) and lambda (nz) of T.
inline void vertical_eigen(int nz, int isym, std::vector<long double> &E, std::vector<long double> &lambda) {
    const long double pi = std::acos(-1.0L);
    E.assign((size_t)nz * nz, 0.0L);
    lambda.assign((size_t)nz, 0.0L);
    for (int q = 0; q < nz; ++q) {
        const long double th = (isym == 1) ? (q + 1.0L) * pi / (nz + 1.0L) : (q + 0.5L) * pi / (nz + 0.5L);
        long double norm = 0.0L;
        for (int k = 0; k < nz; ++k) {
            const long double v = (isym == 1) ? std::sin((k + 1.0L) * th) : std::cos((k + 0.5L) * th);
            E[(size_t)q * nz + k] = v;
            norm += v * v;
        }
        norm = std::sqrt(norm);
        for (int k = 0; k < nz; ++k) E[(size_t)q * nz + k] /= norm;
        lambda[q] = 2.0L - 2.0L * std::cos(th);
    }
}

// T applied to x (the operator the eigen-decomposition diagonalises).
inline void apply_vertical(int nz, int isym, const long double *x, long double *y) {
    for (int k = 0; k < nz; ++k) {
        const long double dn = (k > 0) ? x[k - 1] : 0.0L;
        const long double up = (k + 1 < nz) ? x[k + 1] : 0.0L;
        const long double diag = (k == 0 && isym != 1) ? 1.0L : 2.0L;
        y[k] = diag * x[k] - dn - up;
    }
}

// The radial tridiagonal of one vertical mode q of a slot,
//   lo_j x_{j-1} + (b_j + sigma) x_j + up_j x_{j+1} = v_j,  j = 0 .. n-1
// (b_j FP64, lo_j = up_j = 0 outside the rows: the boundary values are in
// the residual), solved in FP32 by the twisted factorization: side 0
// eliminates rows 0 .. p-1 downwards (x_j + c_j x_{j+1} = g_j), side 1 rows
// n-1 .. p upwards (x_j + e_j x_{j-1} = h_j), p = n / 2; the two meet in the
// 2 x 2 system of rows p-1 and p and substitute back outwards.  Each chain
// is half the radial length.  The values live at y[j * ys] (in place), the
// ratios c_j / e_j at c[j * cs].  Loads of a batch of R rows are issued
// before its recurrence.
struct Radial {
    const double *b;       // [n] diagonal without the shift
    const float *lo, *up;  // [n] sub- and super-diagonal
    double sigma;          // shift of the mode
    int n;
};

BPH_DIRECT_HD float rcp32(float x) {
#if defined(__CUDA_ARCH__)
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return 1.0f / x;
#endif
}

// Side 0 (rows 0 .. p-1, downwards) or side 1 (rows n-1 .. p, upwards).
template <int R>
BPH_DIRECT_HD void twisted_eliminate(const Radial &t, int side, float *y, int ys, float *c, int cs) {
    const int p = t.n / 2;
    const int first = side ? t.n - 1 : 0, count = side ? t.n - p : p, dir = side ? -1 : 1;
    const float *in = side ? t.up : t.lo;   // coupling to the row eliminated before
    const float *out = side ? t.lo : t.up;  // coupling to the row eliminated next
    float ratio = 0.f, val = 0.f;
    for (int i0 = 0; i0 < count; i0 += R) {
        float v[R], a[R], o[R], d[R];
BPH_DIRECT_UNROLL
        for (int u = 0; u < R; ++u) {
            const int j = first + dir * ((i0 + u < count) ? i0 + u : count - 1);
            v[u] = y[j * ys];
            a[u] = (i0 + u > 0) ? in[j] : 0.f;
            o[u] = out[j];
            d[u] = (float)(t.b[j] + t.sigma);
        }
BPH_DIRECT_UNROLL
        for (int u = 0; u < R; ++u) {
            if (i0 + u >= count) break;
            const float r = rcp32(d[u] - a[u] * ratio);
            val = (v[u] - a[u] * val) * r;
            ratio = o[u] * r;
            v[u] = val;
            o[u] = ratio;
        }
BPH_DIRECT_UNROLL
        for (int u = 0; u < R; ++u)
            if (i0 + u < count) {
                const int j = first + dir * (i0 + u);
                y[j * ys] = v[u];
                c[j * cs] = o[u];
            }
    }
}

// The meeting rows p-1 and p after both eliminations: x_{p-1} (side 0) and
// x_p (side 1).  With p = 0 (n = 1) side 1 alone holds the solution.
BPH_DIRECT_HD void twisted_meet(const Radial &t, const float *y, int ys, const float *c, int cs, float &x0, float &x1) {
    const int p = t.n / 2;
    if (p == 0) {
        x0 = 0.f;
        x1 = y[0];
        return;
    }
    const float g = y[(p - 1) * ys], cg = c[(p - 1) * cs], h = y[p * ys], eh = c[p * cs];
    x0 = (g - cg * h) / (1.f - cg * eh);
    x1 = h - eh * x0;
}

// Back substitution of one side from its meeting value, rows p-2 .. 0
// (side 0) or p+1 .. n-1 (side 1); the meeting rows are written apart.
template <int R>
BPH_DIRECT_HD void twisted_substitute(const Radial &t, int side, float x, float *y, int ys, const float *c, int cs) {
    const int p = t.n / 2;
    const int first = side ? p + 1 : p - 2, count = side ? t.n - p - 1 : p - 1, dir = side ? 1 : -1;
    for (int i0 = 0; i0 < count; i0 += R) {
        float v[R], r[R];
BPH_DIRECT_UNROLL
        for (int u = 0; u < R; ++u) {
            const int j = first + dir * ((i0 + u < count) ? i0 + u : count - 1);
            v[u] = y[j * ys];
            r[u] = c[j * cs];
        }
BPH_DIRECT_UNROLL
        for (int u = 0; u < R; ++u) {
            if (i0 + u >= count) break;
            x = v[u] - r[u] * x;
            v[u] = x;
        }
BPH_DIRECT_UNROLL
        for (int u = 0; u < R; ++u)
            if (i0 + u < count) y[(first + dir * (i0 + u)) * ys] = v[u];
    }
}

}  // namespace direct
}  // namespace bph
