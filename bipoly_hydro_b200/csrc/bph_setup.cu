// bph_setup.cu -- setup-time kernels: toroidal-function series
// coefficients, the boundary Green-function tables and the per-step Thomas
// factorisations of the ADI line systems.
//
// This file is compiled with --fmad=false so that the table arithmetic
// rounds like the reference's (no fused multiply-adds); it runs once per
// context and its speed does not matter next to its fidelity.
#include <cmath>

#include "bph_compact.h"
#include "bph_internal.cuh"

namespace bph {
namespace {

// ln Gamma by Lanczos' approximation (gamma = 5, six terms) in the form of
// Numerical Recipes 2nd ed. section 6.1, as gammln.F90:1-30 uses it.  The
// tables depend on this approximation (not on an exact lgamma).
__device__ double d_gammln(double x) {
    const double c[6] = {76.18009172947146, -86.50532032941677, 24.01409824083091,
                         -1.231739572450155, 0.1208650973866179e-2, -0.5395239384953e-5};
    double shifted = x + 5.5;
    double head = (x + 0.5) * log(shifted) - shifted;
    double series = 1.000000000190015;
    double denom = x;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        denom = denom + 1.0;
        series = series + c[i] / denom;
    }
    return head + log(2.5066282746310005 * series / x);
}

// Carlson R_F(0, y, 1) by duplication (Carlson, Numer. Math. 33 (1979)),
// tolerance 0.0025 and the series of rf.F90:19-50.
__device__ double d_rf(double x, double y, double z) {
    double xt = x, yt = y, zt = z, ave, dx, dy, dzz;
    for (int it = 0; it < 200; ++it) {
        double sx = sqrt(xt), sy = sqrt(yt), sz = sqrt(zt);
        double lam = sx * (sy + sz) + sy * sz;
        xt = 0.25 * (xt + lam);
        yt = 0.25 * (yt + lam);
        zt = 0.25 * (zt + lam);
        ave = (1.0 / 3.0) * (xt + yt + zt);
        dx = (ave - xt) / ave;
        dy = (ave - yt) / ave;
        dzz = (ave - zt) / ave;
        if (fmax(fmax(fabs(dx), fabs(dy)), fabs(dzz)) <= 0.0025) break;
    }
    double e2 = dx * dy - dzz * dzz;
    double e3 = dx * dy * dzz;
    return (1.0 + ((1.0 / 24.0) * e2 - 0.1 - (3.0 / 44.0) * e3) * e2 + (1.0 / 14.0) * e3) / sqrt(ave);
}

// Carlson R_D by duplication, tolerance 0.0015, series of rd.F90:20-58.
__device__ double d_rd(double x, double y, double z) {
    const double c1 = 3.0 / 14.0, c2 = 1.0 / 6.0, c3 = 9.0 / 22.0, c4 = 3.0 / 26.0;
    const double c5 = 0.25 * c3, c6 = 1.5 * c4;
    double xt = x, yt = y, zt = z, acc = 0.0, fac = 1.0, ave, dx, dy, dzz;
    for (int it = 0; it < 200; ++it) {
        double sx = sqrt(xt), sy = sqrt(yt), sz = sqrt(zt);
        double lam = sx * (sy + sz) + sy * sz;
        acc = acc + fac / (sz * (zt + lam));
        fac = 0.25 * fac;
        xt = 0.25 * (xt + lam);
        yt = 0.25 * (yt + lam);
        zt = 0.25 * (zt + lam);
        ave = 0.2 * (xt + yt + 3.0 * zt);
        dx = (ave - xt) / ave;
        dy = (ave - yt) / ave;
        dzz = (ave - zt) / ave;
        if (fmax(fmax(fabs(dx), fabs(dy)), fabs(dzz)) <= 0.0015) break;
    }
    double ea = dx * dy, eb = dzz * dzz;
    double ec = ea - eb, ed = ea - 6.0 * eb, ee = ed + ec + ec;
    return 3.0 * acc + fac * (1.0 + ed * (-c1 + c5 * ed - c6 * dzz * ee) +
                              dzz * (c2 * ee + dzz * (-c3 * ec + dzz * c4 * ea))) /
                           (ave * sqrt(ave));
}

// Rolling evaluator of Q for m = 0, 1, 2, ... at one argument x, following
// tm.F90:215-240 (isym 1,2) and tm.F90:289-321 (isym 3): complete elliptic
// integrals plus upward recurrence for x < 1.025, else the 111-term
// hypergeometric series with gammln coefficients.
struct Toroidal {
    bool elliptic;
    double x, q0, q1, log2x, logx;
};

__device__ void tor_init(Toroidal &t, double x, int isym) {
    t.x = x;
    t.elliptic = x < kHyprCutoff;
    if (t.elliptic) {
        double mu = sqrt(2.0 / (1.0 + x));
        double la = sqrt(2.0 * (1.0 + x));
        double q = (1.0 - mu) * (1.0 + mu);
        double rf = d_rf(0.0, q, 1.0);
        double kk = rf;                                               // ellf.F90:16
        double ee = rf - mu * mu * d_rd(0.0, q, 1.0) * 0.3333333333333333;  // elle.F90:16-18
        t.q0 = kk * mu;
        if (isym == 3) {
            const double four_thirds = 4.0 / 3.0, one_third = 1.0 / 3.0;
            t.q1 = (four_thirds * x * x - one_third) * mu * kk - four_thirds * x * la * ee;
        } else {
            t.q1 = x * mu * kk - la * ee;
        }
    } else {
        t.log2x = log(2.0 * x);
        t.logx = log(x);
    }
}

// qc layout: coefh[mmax], nu[mmax], dcoefh[mmax][111].
__device__ double tor_next(Toroidal &t, int m, const double *__restrict__ qc, int mmax, int isym) {
    if (t.elliptic) {
        if (m == 0) return t.q0;
        if (m == 1) return t.q1;
        double nu = qc[mmax + m], x = t.x, qn;
        if (isym == 3) {
            qn = t.q1 * ((2.0 * nu + 3.0) * (2.0 * nu + 1.0) * x * x / ((nu + 2.0) * (nu + 1.0)) -
                         (2.0 * nu + 3.0) * nu * nu / ((2.0 * nu - 1.0) * (nu + 2.0) * (nu + 1.0)) -
                         (nu + 1.0) / (nu + 2.0)) -
                 t.q0 * (2.0 * nu + 3.0) * (nu - 1.0) * nu / ((2.0 * nu - 1.0) * (nu + 2.0) * (nu + 1.0));
        } else {
            qn = (2.0 * nu + 1.0) / (nu + 1.0) * x * t.q1 - nu / (nu + 1.0) * t.q0;
        }
        t.q0 = t.q1;
        t.q1 = qn;
        return qn;
    }
    double expo = (isym == 3) ? (2.0 * (double)m + 0.5) : ((double)m + 0.5);
    double pref = exp(qc[m] - expo * t.log2x);
    const double *dc = qc + 2 * mmax + m * (kHyprUprBnd + 1);
    double acc = 0.0, ri = 0.0;
    for (int ir = 0; ir <= kHyprUprBnd; ++ir) {
        acc = acc + exp(__ldg(dc + ir) - 2.0 * ri * t.logx);
        ri = ri + 1.0;
    }
    return pref * acc;
}

// Series coefficients (tm.F90:105-155): one thread per (m, ir).
__global__ void k_qcoef(double *qc, int mmax, int isym) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mmax * (kHyprUprBnd + 1)) return;
    int m = t / (kHyprUprBnd + 1), ir = t % (kHyprUprBnd + 1);
    double mm = (isym == 3) ? 2.0 * (double)m : (double)m;
    double aa = 0.5 * (mm + 1.5), bb = 0.5 * (mm + 0.5), cc = mm + 1.0;
    double ri = (double)ir;
    qc[2 * mmax + m * (kHyprUprBnd + 1) + ir] =
        d_gammln(aa + ri) + d_gammln(bb + ri) - d_gammln(cc + ri) - d_gammln(ri + 1.0);
    if (ir == 0) {
        qc[m] = d_gammln(0.5) + d_gammln(mm + 0.5) - d_gammln(aa) - d_gammln(bb);
        // nu(m) = index - 2.5 (or 2*index - 4.5 for isym 3), index = m+1 (1-based m).
        double idx = (double)(m + 1);
        qc[mmax + m] = (m >= 2) ? ((isym == 3) ? 2.0 * idx - 4.5 : idx - 2.5) : 0.0;
    }
}

// Green tables (tm.F90:157-363, sm.F90:172-382, bm.F90:130-172): one thread
// per (source zone p, boundary row b); G[m][b][p] for all m.
__global__ void k_green_tables(const double *__restrict__ grid, const double *__restrict__ qc,
                               double *__restrict__ G, int numr, int numz, int nr, int nz, int nb,
                               int mmax, int isym, double piinv) {
    long long np = (long long)nr * nz;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np * nb) return;
    const double *rhf = grid, *rhfinv = grid + numr, *zhf = grid + 2 * numr;
    int p = (int)(t % np), b = (int)(t / np);
    int jl = p % nr + 2, kl = p / nr + 2;
    double rs = rhf[jl - 1], rsinv = rhfinv[jl - 1], zs = zhf[kl - 1];
    double rb, rbinv, zb;
    bool img = (isym != 1);
    if (b < nr) {
        int jg = b + 2;
        rb = rhf[jg - 1];
        rbinv = rhfinv[jg - 1];
        zb = zhf[numz - 1];
    } else if (b < nr + nz) {
        int kg = b - nr + 2;
        rb = rhf[numr - 1];
        rbinv = 1.0 / rb;
        zb = zhf[kg - 1];
    } else {
        int jg = b - nr - nz + 2;
        rb = rhf[jg - 1];
        rbinv = rhfinv[jg - 1];
        zb = zhf[0];
        img = false;
    }
    double coef = sqrt(rs * rbinv) * piinv;
    double dmi = zb - zs, dpl = zb + zs;
    double xm = (isym != 1) ? 0.5 * rsinv * rbinv * (dmi * dmi + rs * rs + rb * rb)
                            : 0.5 * rsinv * rbinv * (dmi * dmi + rb * rb + rs * rs);
    Toroidal tm_, tp_;
    tor_init(tm_, xm, isym);
    if (img) tor_init(tp_, 0.5 * rsinv * rbinv * (dpl * dpl + rs * rs + rb * rb), isym);
    double *out = G + (long long)b * np + p;
    const long long mstride = (long long)nb * np;
    for (int m = 0; m < mmax; ++m) {
        double qm = tor_next(tm_, m, qc, mmax, isym);
        double v;
        if (img) {
            double qp = tor_next(tp_, m, qc, mmax, isym);
            v = coef * (qp + qm);
        } else {
            v = coef * qm;
        }
        out[m * mstride] = v;
    }
}

// Compact tables (bph_compact.h).  Tiles of the top (set 0) and bottom
// (set 1, isym 1) rows: one thread per (set, tile, height k, element);
// element (r, c) of tile (I, J) is H(jb = 8I + r, j = 8J + c, k) =
// G(jb, j, k) / r_j with G as k_green_tables forms it; zero outside the
// nr x nr plane and at the padding heights k >= nz.  Layout
// [m][set][k < nzp][tile][64]: at one height the tiles are contiguous, so
// the contraction's warps read neighbouring 512-byte tiles.
__global__ void k_green_compact_tiles(const double *__restrict__ grid, const double *__restrict__ qc,
                                      double *__restrict__ T, int numr, int numz, int nr, int nz, int nzp, int nb8,
                                      int npair, int nsets, int mmax, int isym, double piinv) {
    const long long per_m = (long long)nsets * npair * nzp * 64;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per_m) return;
    const double *rhf = grid, *rhfinv = grid + numr, *zhf = grid + 2 * numr;
    const int e = (int)(t % 64);
    long long rest = t / 64;
    const int q = (int)(rest % npair);
    rest /= npair;
    const int k = (int)(rest % nzp), set = (int)(rest / nzp);
    int I, J;
    compact::pair_blocks(q, nb8, &I, &J);
    const int jb = 8 * I + (e >> 3), j = 8 * J + (e & 7);
    double *out = T + t;
    if (jb >= nr || j >= nr || k >= nz) {
        for (int m = 0; m < mmax; ++m) out[m * per_m] = 0.0;
        return;
    }
    const double rs = rhf[j + 1], rsinv = rhfinv[j + 1], zs = zhf[k + 1];
    const double rb = rhf[jb + 1], rbinv = rhfinv[jb + 1];
    const double zb = (set == 0) ? zhf[numz - 1] : zhf[0];
    const bool img = (set == 0) && (isym != 1);
    const double coef = sqrt(rs * rbinv) * piinv;
    const double dmi = zb - zs, dpl = zb + zs;
    const double xm = (isym != 1) ? 0.5 * rsinv * rbinv * (dmi * dmi + rs * rs + rb * rb)
                                  : 0.5 * rsinv * rbinv * (dmi * dmi + rb * rb + rs * rs);
    Toroidal tm_, tp_;
    tor_init(tm_, xm, isym);
    if (img) tor_init(tp_, 0.5 * rsinv * rbinv * (dpl * dpl + rs * rs + rb * rb), isym);
    for (int m = 0; m < mmax; ++m) {
        const double qm = tor_next(tm_, m, qc, mmax, isym);
        double v;
        if (img) {
            const double qp = tor_next(tp_, m, qc, mmax, isym);
            v = coef * (qp + qm);
        } else {
            v = coef * qm;
        }
        out[m * per_m] = v * rsinv;
    }
}

// Side vectors: one thread per (radial zone j, position in U or V).
// U_j(d), d = kb - k in [-(nz-1), nz-1], is evaluated at the pair
// (kb, k) = (|d|, 0); V_j(s), s = kb + k in [0, 2 nz - 2], at
// (min(s, nz-1), s - min(s, nz-1)); both zero-padded to `stride`.
// Layout [m][j][U | V][stride].
__global__ void k_green_compact_side(const double *__restrict__ grid, const double *__restrict__ qc,
                                     double *__restrict__ Sd, int numr, int nr, int nz, int stride, int mmax,
                                     int isym, double piinv) {
    const long long per_m = (long long)nr * 2 * stride;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per_m) return;
    const double *rhf = grid, *rhfinv = grid + numr, *zhf = grid + 2 * numr;
    const int pos = (int)(t % stride);
    const int which = (int)((t / stride) % 2);  // 0: U, 1: V
    const int j = (int)(t / (2LL * stride));
    double *out = Sd + t;
    int kb, k;
    bool valid;
    if (which == 0) {
        const int d = pos - (nz - 1);
        kb = d < 0 ? -d : d;
        k = 0;
        valid = pos <= 2 * nz - 2;
    } else {
        kb = pos < nz - 1 ? pos : nz - 1;
        k = pos - kb;
        valid = (isym != 1) && pos <= 2 * nz - 2;
    }
    if (!valid) {
        for (int m = 0; m < mmax; ++m) out[m * per_m] = 0.0;
        return;
    }
    const double rs = rhf[j + 1], rsinv = rhfinv[j + 1], zs = zhf[k + 1];
    const double rb = rhf[numr - 1], rbinv = 1.0 / rb;
    const double zb = zhf[kb + 1];
    const double coef = sqrt(rs * rbinv) * piinv;
    double x;
    if (which == 0) {
        const double dmi = zb - zs;
        x = (isym != 1) ? 0.5 * rsinv * rbinv * (dmi * dmi + rs * rs + rb * rb)
                        : 0.5 * rsinv * rbinv * (dmi * dmi + rb * rb + rs * rs);
    } else {
        const double dpl = zb + zs;
        x = 0.5 * rsinv * rbinv * (dpl * dpl + rs * rs + rb * rb);
    }
    Toroidal tq;
    tor_init(tq, x, isym);
    for (int m = 0; m < mmax; ++m) out[m * per_m] = coef * tor_next(tq, m, qc, mmax, isym);
}

// Thomas factorisations for one ADI schedule (tridagr.F90:41-60,
// tridagz.F90:115-132).  Radial: one thread per (step, slot); vertical: one
// thread per step.  For a line of n unknowns, five arrays of n:
//   f[0] = 1/bet_j, f[1] = a_j/bet_j, f[2] = gam_j     (Thomas:
//     y_j = w_j/bet_j - (a_j/bet_j) y_{j-1},  x_j = y_j - gam_{j+1} x_{j+1})
//   f[3] = forward carry  G_j = prod_{i=s..j} (-a_i/bet_i)
//   f[4] = backward carry K_j = prod_{i=j+1..e+1} (-gam_i), gam_n = 0
// with [s, e] the kAdiSeg-long segment holding j: a segment solved with a
// zero carry-in gives L (or M), and the true values are L + G y_{s-1}
// (or M + K x_{e+1}).
__device__ void line_carries(double *f, int n) {
    double *dd = f + n, *gam = f + 2 * n, *G = f + 3 * n, *K = f + 4 * n;
    for (int s0 = 0; s0 < n; s0 += kAdiSeg) {
        int e0 = min(s0 + kAdiSeg, n) - 1;
        double g = 1.0;
        for (int j = s0; j <= e0; ++j) {
            g = -dd[j] * g;
            G[j] = g;
        }
        double k = 1.0;
        for (int j = e0; j >= s0; --j) {
            double gnext = (j + 1 < n) ? gam[j + 1] : 0.0;
            k = -gnext * k;
            K[j] = k;
        }
    }
}

__global__ void k_adi_factors(const double *__restrict__ dt, int nsteps, const double *__restrict__ brb,
                              const double *__restrict__ alphar, const double *__restrict__ betar,
                              const double *__restrict__ bzb, double gamma, double *__restrict__ rad,
                              double *__restrict__ ver, int numr, int numz, int N) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nr = numr - 2, nz = numz - 2;
    if (t < nsteps * N) {
        int step = t / N, s = t % N;
        double dtt = dt[step];
        const double *b = brb + (long long)s * numr;
        double *o = rad + ((long long)step * N + s) * kAdiFactors * nr;
        double bet = b[1] + dtt;  // J = 2
        o[0] = 1.0 / bet;
        o[nr] = 0.0;
        o[2 * nr] = 0.0;
        for (int j = 1; j < nr; ++j) {
            int J = j + 2;
            double gam = alphar[J - 2] / bet;
            bet = (b[J - 1] + dtt) - betar[J - 1] * gam;
            double ib = 1.0 / bet;
            o[j] = ib;
            o[nr + j] = betar[J - 1] * ib;
            o[2 * nr + j] = gam;
        }
        line_carries(o, nr);
    } else if (t < nsteps * N + nsteps) {
        int step = t - nsteps * N;
        double dtt = dt[step];
        const double az = -gamma, cz = -gamma;
        double *o = ver + (long long)step * kAdiFactors * nz;
        double bet = bzb[1] + dtt;  // K = 2
        o[0] = 1.0 / bet;
        o[nz] = 0.0;
        o[2 * nz] = 0.0;
        for (int k = 1; k < nz; ++k) {
            int K = k + 2;
            double gam = cz / bet;
            bet = (bzb[K - 1] + dtt) - az * gam;
            double ib = 1.0 / bet;
            o[k] = ib;
            o[nz + k] = az * ib;
            o[2 * nz + k] = gam;
        }
        line_carries(o, nz);
    }
}

}  // namespace

cudaError_t launch_qcoef(bph_ctx *c) {
    int n = c->g.mmax * (kHyprUprBnd + 1);
    k_qcoef<<<(n + 127) / 128, 128, 0, c->stream>>>(c->d_qcoef, c->g.mmax, c->g.isym);
    ++c->launches;
    return cudaGetLastError();
}

cudaError_t launch_green_tables(bph_ctx *c) {
    long long n = c->np * c->nb;
    int threads = 128;
    long long blocks = (n + threads - 1) / threads;
    k_green_tables<<<(unsigned)blocks, threads, 0, c->stream>>>(c->d_grid, c->d_qcoef, c->d_green, c->g.numr,
                                                                c->g.numz, c->nr, c->nz, c->nb, c->g.mmax,
                                                                c->g.isym, 1.0 / c->pi);
    ++c->launches;
    return cudaGetLastError();
}

cudaError_t launch_green_compact(bph_ctx *c) {
    const compact::Dims d = compact::dims(c->nr, c->nz, c->g.isym);
    const int threads = 128;
    const long long nt = (long long)d.nsets * d.npair * d.nzp * 64;
    k_green_compact_tiles<<<(unsigned)((nt + threads - 1) / threads), threads, 0, c->stream>>>(
        c->d_grid, c->d_qcoef, c->d_gtile, c->g.numr, c->g.numz, c->nr, c->nz, d.nzp, d.nb8, d.npair, d.nsets,
        c->g.mmax, c->g.isym, 1.0 / c->pi);
    const long long ns = (long long)c->nr * 2 * d.stride;
    k_green_compact_side<<<(unsigned)((ns + threads - 1) / threads), threads, 0, c->stream>>>(
        c->d_grid, c->d_qcoef, c->d_gside, c->g.numr, c->nr, c->nz, d.stride, c->g.mmax, c->g.isym, 1.0 / c->pi);
    c->launches += 2;
    return cudaGetLastError();
}

// One thread per (step, line system): the [ib, dd, gam, G, K] arrays of
// k_adi_factors rearranged into packed_block<T> layout (pairs (G_j, gam_{j+1})).
template <typename T>
__global__ void k_pack_factors(const double *__restrict__ rad, const double *__restrict__ ver,
                               T *__restrict__ rad_pk, T *__restrict__ ver_pk, int nsteps, int N, int nr, int nz) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nrad = (long long)nsteps * N;
    if (t >= nrad + nsteps) return;
    const bool radial = t < nrad;
    const int n = radial ? nr : nz;
    const double *src = radial ? rad + t * kAdiFactors * nr : ver + (t - nrad) * kAdiFactors * nz;
    const int pb = packed_block<T>(n);
    T *dst = radial ? rad_pk + t * pb : ver_pk + (t - nrad) * pb;
    for (int j = 0; j < n; ++j) {
        dst[j] = (T)src[j];
        dst[n + j] = (T)src[n + j];
        dst[2 * n + 2 * j] = (T)src[3 * n + j];
        dst[2 * n + 2 * j + 1] = (T)((j + 1 < n) ? src[2 * n + j + 1] : 0.0);
        dst[4 * n + j] = (T)src[4 * n + j];
    }
    for (int j = 5 * n; j < pb; ++j) dst[j] = (T)0;
}

cudaError_t launch_pack_factors(bph_ctx *c, Schedule &s) {
    const long long n = (long long)s.nsteps * c->N + s.nsteps;
    const unsigned blocks = (unsigned)((n + 127) / 128);
    k_pack_factors<double><<<blocks, 128, 0, c->stream>>>(s.d_rad, s.d_ver, (double *)s.d_rad_pk[0],
                                                          (double *)s.d_ver_pk[0], s.nsteps, c->N, c->nr, c->nz);
    k_pack_factors<float><<<blocks, 128, 0, c->stream>>>(s.d_rad, s.d_ver, (float *)s.d_rad_pk[1],
                                                         (float *)s.d_ver_pk[1], s.nsteps, c->N, c->nr, c->nz);
    c->launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_adi_factors(bph_ctx *c, Schedule &s) {
    int n = s.nsteps * c->N + s.nsteps;
    k_adi_factors<<<(n + 127) / 128, 128, 0, c->stream>>>(s.d_dt, s.nsteps, c->d_brb, c->d_alphar, c->d_betar,
                                                          c->d_bzb, c->gamma, s.d_rad, s.d_ver, c->g.numr,
                                                          c->g.numz, c->N);
    ++c->launches;
    return cudaGetLastError();
}

}  // namespace bph
