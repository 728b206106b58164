/*
 * bph_oracle.c -- CPU restatement (FP64, one MPI rank) of bipoly_hydro's
 * self-gravity Poisson solve.  TEST INFRASTRUCTURE ONLY: the parity checker
 * and the timed CPU baseline; never part of the product path.
 *
 * Parity UNPINNED by the reference itself (no golden vectors exist and the
 * Fortran cannot be compiled in this image); pinned by analytic known
 * answers in tests/test_oracle_*.py.
 *
 * With one rank every MPI transpose (swap_phi_r, swap_r_phi, swap_r_z,
 * swap_z_r) is a copy, every halo exchange (comm, comm_r_sweep,
 * comm_z_sweep) a no-op and every mpi_reduce in bessel.F90:305-394 the
 * identity, so they do not appear below.
 *
 * Arithmetic follows the reference's expression order (compile with
 * -ffp-contract=off) so that the only differences from the Fortran are the
 * libm's last-bit rounding.
 */
#include "bph_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HYPR_CUTOFF 1.025   /* pot.h:5 */
#define HYPR_UPR_BND 110    /* pot.h:7 */

static __thread char g_err[256];
static void set_err(const char *msg) { snprintf(g_err, sizeof g_err, "%s", msg); }
const char *orc_last_error(void) { return g_err; }

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

struct orc_ctx {
    orc_grid g;
    int nr, nz, nb;            /* interior radial / vertical sizes, boundary rows */
    long nplane, ntot;
    double pi, dz, dphi, drinv, dzinv, dphiinv, gamma, piinv, four_pi, factor;
    double *r_g, *rhf_g, *rinv_g, *rhfinv_g, *zhf_g;   /* [numr]/[numz], index J-1 */
    double *bes_cos, *bes_sin;                         /* [mmax][numphi] */
    int *mode;                                         /* [numphi] */
    double *elm, *m1mode;                              /* [numphi] */
    double *alphar, *betar, *alphaz, *betaz;           /* [numr] */
    double *brb, *elambdazb;                           /* [numphi][numr] */
    double *bzb;                                       /* [numz] */
    double az, cz;
    double *green;                                     /* [mmax][nb][nr*nz] */
    double *S;                                         /* [mmax][nb][2] */
    const double *S_override;                          /* test hook: boundary moments to use instead */
    double *potp, *rhop;                               /* [numphi][numz][numr] */
};

#define IX(c, J, K, L) ((long)((J) - 1) + (long)(c)->g.numr * ((long)((K) - 1) + (long)(c)->g.numz * (long)((L) - 1)))

/* ------------------------------------------------------------------ */
/* Special functions                                                   */
/* ------------------------------------------------------------------ */

/* ln Gamma(x), x > 0, by Lanczos' approximation with gamma = 5 and six
 * series terms in the form Numerical Recipes 2nd ed. section 6.1 publishes
 * (gammln.F90:1-30).  The tables need this approximation, not lgamma():
 * it differs from lgamma by up to ~2e-10. */
double orc_gammln(double x) {
    static const double lanczos_c[6] = {
        76.18009172947146, -86.50532032941677, 24.01409824083091,
        -1.231739572450155, 0.1208650973866179e-2, -0.5395239384953e-5};
    const double sqrt_two_pi = 2.5066282746310005;
    double shifted = x + 5.5;
    double head = (x + 0.5) * log(shifted) - shifted;
    double series = 1.000000000190015;
    double denom = x;
    for (int i = 0; i < 6; ++i) {
        denom = denom + 1.0;
        series = series + lanczos_c[i] / denom;
    }
    return head + log(sqrt_two_pi * series / x);
}

/* Carlson's symmetric integral R_F(x,y,z) by the duplication theorem
 * (B. C. Carlson, Numer. Math. 33 (1979) 1-16), stopping tolerance 0.0025
 * and the fifth-order series of rf.F90:19-50.  Invalid arguments give NaN
 * (the reference STOPs, rf.F90:27-30). */
double orc_rf(double x, double y, double z) {
    const double tol = 0.0025, tiny = 2.0e-307, big = 2.0e307;
    double mn = fmin(fmin(x, y), z), mx = fmax(fmax(x, y), z);
    double mpair = fmin(fmin(x + y, x + z), y + z);
    if (mn < 0.0 || mpair < tiny || mx > big) return NAN;
    double xt = x, yt = y, zt = z, ave, dx, dy, dzz;
    for (;;) {
        double sx = sqrt(xt), sy = sqrt(yt), sz = sqrt(zt);
        double lam = sx * (sy + sz) + sy * sz;
        xt = 0.25 * (xt + lam);
        yt = 0.25 * (yt + lam);
        zt = 0.25 * (zt + lam);
        ave = (1.0 / 3.0) * (xt + yt + zt);
        dx = (ave - xt) / ave;
        dy = (ave - yt) / ave;
        dzz = (ave - zt) / ave;
        if (fmax(fmax(fabs(dx), fabs(dy)), fabs(dzz)) <= tol) break;
    }
    double e2 = dx * dy - dzz * dzz;
    double e3 = dx * dy * dzz;
    return (1.0 + ((1.0 / 24.0) * e2 - 0.1 - (3.0 / 44.0) * e3) * e2 + (1.0 / 14.0) * e3) / sqrt(ave);
}

/* Carlson's R_D(x,y,z) by duplication (Carlson 1979), tolerance 0.0015 and
 * the series of rd.F90:20-58.  Invalid arguments give NaN. */
double orc_rd(double x, double y, double z) {
    const double tol = 0.0015, tiny = 1.0e-204, big = 1.0e201;
    const double c1 = 3.0 / 14.0, c2 = 1.0 / 6.0, c3 = 9.0 / 22.0, c4 = 3.0 / 26.0;
    const double c5 = 0.25 * c3, c6 = 1.5 * c4;
    if (fmin(x, y) < 0.0 || fmin(x + y, z) < tiny || fmax(fmax(x, y), z) > big) return NAN;
    double xt = x, yt = y, zt = z, acc = 0.0, fac = 1.0, ave, dx, dy, dzz;
    for (;;) {
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
        if (fmax(fmax(fabs(dx), fabs(dy)), fabs(dzz)) <= tol) break;
    }
    double ea = dx * dy, eb = dzz * dzz;
    double ec = ea - eb, ed = ea - 6.0 * eb, ee = ed + ec + ec;
    return 3.0 * acc + fac * (1.0 + ed * (-c1 + c5 * ed - c6 * dzz * ee) +
                              dzz * (c2 * ee + dzz * (-c3 * ec + dzz * c4 * ea))) /
                           (ave * sqrt(ave));
}

/* Complete K(k) = R_F(0, 1-k^2, 1) (ellf.F90:16). */
double orc_ellf(double k) { return orc_rf(0.0, (1.0 - k) * (1.0 + k), 1.0); }

/* Complete E(k) = R_F - k^2 R_D / 3 (elle.F90:16-18). */
double orc_elle(double k) {
    double q = (1.0 - k) * (1.0 + k);
    return orc_rf(0.0, q, 1.0) - k * k * orc_rd(0.0, q, 1.0) * 0.3333333333333333;
}

/* Series coefficients of tm.F90:105-155 (same in sm.F90, bm.F90):
 * nu[m] for the upward recurrence, coefh[m] = ln of the hypergeometric
 * prefactor, dcoefh[m][ir] = ln of the ir-th series term coefficient. */
typedef struct {
    int mmax, isym;
    double *nu, *coefh, *dcoefh; /* dcoefh[m*(HYPR_UPR_BND+1)+ir] */
} qcoef_t;

static void qcoef_init(qcoef_t *qc, int isym, int mmax) {
    qc->mmax = mmax;
    qc->isym = isym;
    qc->nu = calloc((size_t)mmax, sizeof(double));
    qc->coefh = calloc((size_t)mmax, sizeof(double));
    qc->dcoefh = calloc((size_t)mmax * (HYPR_UPR_BND + 1), sizeof(double));
    double gl_half = orc_gammln(0.5);
    double idx = 3.0;
    for (int m = 2; m < mmax; ++m) {
        qc->nu[m] = (isym == 3) ? 2.0 * idx - 4.5 : idx - 2.5;
        idx = idx + 1.0;
    }
    idx = 1.0;
    for (int m = 0; m < mmax; ++m) {
        double mm = (isym == 3) ? 2.0 * (idx - 1.0) : idx - 1.0;
        double aa = 0.5 * (mm + 1.5), bb = 0.5 * (mm + 0.5), cc = mm + 1.0;
        qc->coefh[m] = gl_half + orc_gammln(mm + 0.5) - orc_gammln(aa) - orc_gammln(bb);
        double ri = 0.0;
        for (int ir = 0; ir <= HYPR_UPR_BND; ++ir) {
            qc->dcoefh[m * (HYPR_UPR_BND + 1) + ir] =
                orc_gammln(aa + ri) + orc_gammln(bb + ri) - orc_gammln(cc + ri) - orc_gammln(ri + 1.0);
            ri = ri + 1.0;
        }
        idx = idx + 1.0;
    }
}

static void qcoef_free(qcoef_t *qc) {
    free(qc->nu);
    free(qc->coefh);
    free(qc->dcoefh);
}

/* Q for one argument x >= 1, m = 0..mmax-1: elliptic integrals plus upward
 * recurrence for x < 1.025, else the 111-term hypergeometric series
 * (tm.F90:215-240 for isym 1,2; tm.F90:289-321 for isym 3). */
static void toroidal_eval(const qcoef_t *qc, double x, double *q) {
    const int mmax = qc->mmax;
    if (x < HYPR_CUTOFF) {
        double mu = sqrt(2.0 / (1.0 + x));
        double la = sqrt(2.0 * (1.0 + x));
        double kk = orc_ellf(mu), ee = orc_elle(mu);
        q[0] = kk * mu;
        if (qc->isym == 3) {
            const double four_thirds = 4.0 / 3.0, one_third = 1.0 / 3.0;
            if (mmax > 1) q[1] = (four_thirds * x * x - one_third) * mu * kk - four_thirds * x * la * ee;
            for (int m = 2; m < mmax; ++m) {
                double nu = qc->nu[m];
                q[m] = q[m - 1] * ((2.0 * nu + 3.0) * (2.0 * nu + 1.0) * x * x / ((nu + 2.0) * (nu + 1.0)) -
                                   (2.0 * nu + 3.0) * nu * nu / ((2.0 * nu - 1.0) * (nu + 2.0) * (nu + 1.0)) -
                                   (nu + 1.0) / (nu + 2.0)) -
                       q[m - 2] * (2.0 * nu + 3.0) * (nu - 1.0) * nu / ((2.0 * nu - 1.0) * (nu + 2.0) * (nu + 1.0));
            }
        } else {
            if (mmax > 1) q[1] = x * mu * kk - la * ee;
            for (int m = 2; m < mmax; ++m) {
                double nu = qc->nu[m];
                q[m] = (2.0 * nu + 1.0) / (nu + 1.0) * x * q[m - 1] - nu / (nu + 1.0) * q[m - 2];
            }
        }
    } else {
        /* The logs are pure functions of x, so evaluating them once per
         * argument gives the same values as the reference's per-term
         * alog() calls. */
        double log2x = log(2.0 * x), logx = log(x);
        double idx = (qc->isym == 3) ? 1.0 : 0.0;
        for (int m = 0; m < mmax; ++m) {
            double expo = (qc->isym == 3) ? (2.0 * (idx - 1.0) + 0.5) : (idx + 0.5);
            double pref = exp(qc->coefh[m] - expo * log2x);
            double acc = 0.0, ri = 0.0;
            const double *dc = qc->dcoefh + (long)m * (HYPR_UPR_BND + 1);
            for (int ir = 0; ir <= HYPR_UPR_BND; ++ir) {
                acc = acc + exp(dc[ir] - 2.0 * ri * logx);
                ri = ri + 1.0;
            }
            q[m] = pref * acc;
            idx = idx + 1.0;
        }
    }
}

void orc_toroidal(double x, int isym, int mmax, double *q) {
    qcoef_t qc;
    qcoef_init(&qc, isym, mmax);
    toroidal_eval(&qc, x, q);
    qcoef_free(&qc);
}

/* ------------------------------------------------------------------ */
/* Azimuthal real FFT (realft.F90)                                     */
/* ------------------------------------------------------------------ */

/* In-place complex radix-2 FFT of nn complex values stored interleaved
 * (re, im) at data[0..2nn-1] with element stride `stride`: bit reversal,
 * then Danielson-Lanczos passes with a trigonometric recurrence for the
 * twiddles (four1, realft.F90:83-150).  The reference's 2*pi constant is
 * the literal 6.28318530717959, kept here. */
static void four1_col(double *d, long s, int nn, int isign) {
    int n = 2 * nn;
    int j = 0;
    for (int i = 0; i < n; i += 2) {
        if (j > i) {
            double tr = d[s * j], ti = d[s * (j + 1)];
            d[s * j] = d[s * i];
            d[s * (j + 1)] = d[s * (i + 1)];
            d[s * i] = tr;
            d[s * (i + 1)] = ti;
        }
        int m = n / 2;
        while (m >= 2 && j >= m) {
            j -= m;
            m /= 2;
        }
        j += m;
    }
    int span = 2;
    while (n > span) {
        int istep = 2 * span;
        double theta = 6.28318530717959 / (double)(isign * span);
        double sh = sin(0.5 * theta);
        double wpr = -2.0 * (sh * sh);
        double wpi = sin(theta);
        double wr = 1.0, wi = 0.0;
        for (int m = 0; m < span; m += 2) {
            for (int i = m; i < n; i += istep) {
                int jj = i + span;
                double tr = wr * d[s * jj] - wi * d[s * (jj + 1)];
                double ti = wr * d[s * (jj + 1)] + wi * d[s * jj];
                d[s * jj] = d[s * i] - tr;
                d[s * (jj + 1)] = d[s * (i + 1)] - ti;
                d[s * i] = d[s * i] + tr;
                d[s * (i + 1)] = d[s * (i + 1)] + ti;
            }
            double wt = wr;
            wr = wr * wpr - wi * wpi + wr;
            wi = wi * wpr + wt * wpi + wi;
        }
        span = istep;
    }
}

/* Real FFT of n points (realft.F90:5-77).  isign=+1: forward, giving
 * d[0]=F_0, d[1]=F_{n/2}, d[2k],d[2k+1] = Re,Im F_k with
 * F_k = sum_l f_l exp(+2 pi i k l / n).  isign=-1: the inverse times n/2. */
void orc_realft(double *d, long s, int n, int isign) {
    double theta = 3.141592653589793 / (double)(n / 2);
    double c1 = 0.5, c2;
    if (isign == 1) {
        c2 = -0.5;
        four1_col(d, s, n / 2, +1);
    } else {
        c2 = 0.5;
        theta = -theta;
    }
    double sh = sin(0.5 * theta);
    double wpr = -2.0 * (sh * sh);
    double wpi = sin(theta);
    double wr = 1.0 + wpr, wi = wpi;
    int n2p3 = n + 3;
    for (int i = 2; i <= n / 4; ++i) {
        int i1 = 2 * i - 1, i2 = i1 + 1, i3 = n2p3 - i2, i4 = i3 + 1; /* 1-based */
        double *p1 = d + s * (i1 - 1), *p2 = d + s * (i2 - 1), *p3 = d + s * (i3 - 1), *p4 = d + s * (i4 - 1);
        double wrs = wr, wis = wi;
        double h1r = c1 * (*p1 + *p3);
        double h1i = c1 * (*p2 - *p4);
        double h2r = -(c2 * (*p2 + *p4));
        double h2i = c2 * (*p1 - *p3);
        *p1 = h1r + wrs * h2r - wis * h2i;
        *p2 = h1i + wrs * h2i + wis * h2r;
        *p3 = h1r - wrs * h2r + wis * h2i;
        *p4 = -h1i + wrs * h2i + wis * h2r;
        double wt = wr;
        wr = wr * wpr - wi * wpi + wr;
        wi = wi * wpr + wt * wpi + wi;
    }
    double h1r = d[0];
    if (isign == 1) {
        d[0] = h1r + d[s];
        d[s] = h1r - d[s];
    } else {
        d[0] = c1 * (h1r + d[s]);
        d[s] = c1 * (h1r - d[s]);
        four1_col(d, s, n / 2, -1);
    }
}

/* ------------------------------------------------------------------ */
/* Setup (setup_frac.F90:374-463, potsetup.F90, tm/sm/bm)              */
/* ------------------------------------------------------------------ */

int orc_num_boundary_rows(const orc_ctx *c) { return c->nb; }
const double *orc_green(const orc_ctx *c) { return c->green; }
const double *orc_moments_S(const orc_ctx *c) { return c->S; }
int orc_slot_mode(const orc_ctx *c, int slot0) { return c->mode[slot0]; }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* Global grid (setup_frac.F90:374-463), one rank so local == global. */
static void grid_init(orc_ctx *c) {
    const orc_grid *g = &c->g;
    c->pi = acos(-1.0);
    c->dz = g->dr;
    c->dphi = 2.0 * c->pi * (1.0 / (double)g->numphi);
    c->drinv = 1.0 / g->dr;
    c->dzinv = 1.0 / c->dz;
    c->dphiinv = 1.0 / c->dphi;
    double x = 1.0;
    for (int J = 1; J <= g->numr; ++J) {
        c->r_g[J - 1] = (x - 2.0) * g->dr;
        x = x + 1.0;
    }
    for (int J = 1; J <= g->numr; ++J) {
        c->rhf_g[J - 1] = c->r_g[J - 1] + 0.5 * g->dr;
        c->rinv_g[J - 1] = (c->r_g[J - 1] != 0.0) ? 1.0 / c->r_g[J - 1] : 0.0;
        c->rhfinv_g[J - 1] = 1.0 / c->rhf_g[J - 1];
    }
    x = 1.0;
    double offset = (g->isym != 1) ? 0.0 : -(double)(g->numz / 2) * c->dz;
    for (int K = 1; K <= g->numz; ++K) {
        c->zhf_g[K - 1] = (g->isym != 1) ? (x - 1.5) * c->dz : offset + (x - 0.5) * c->dz;
        x = x + 1.0;
    }
}

/* Green tables (tm.F90:157-363, sm.F90:172-382, bm.F90:130-172).  For a
 * source zone p=(jl,kl) and a boundary point at (rb, zb):
 *   G = sqrt(rhf(jl)/rb)/pi * [Q(chi-) (+ Q(chi+) for isym 2,3)],
 *   chi-+ = ((zb -+ z')^2 + r'^2 + rb^2) / (2 r' rb).
 * `order` reproduces the reference's term order inside chi:
 *   0: (dz^2 + rhf(jl)^2 + rb^2)   tm/sm isym 2,3 and their chi+ terms
 *   1: (dz^2 + rb^2 + rhf(jl)^2)   tm isym 1, bm, sm isym 1 */
static void green_row(const orc_ctx *c, const qcoef_t *qc, double rb, double rbinv, double zb, int top_like,
                      int with_image, int order, int b) {
    const orc_grid *g = &c->g;
    const int nr = c->nr, nz = c->nz, mmax = g->mmax;
    const long np = (long)nr * nz;
    double qp[64], qm[64];
    for (int kl = 2; kl <= g->numz - 1; ++kl) {
        for (int jl = 2; jl <= g->numr - 1; ++jl) {
            double rs = c->rhf_g[jl - 1], rsinv = c->rhfinv_g[jl - 1], zs = c->zhf_g[kl - 1];
            double coef = sqrt(rs * rbinv) * c->piinv;
            double dmi = zb - zs, dpl = zb + zs;
            double xm, xp = 0.0;
            if (order == 0)
                xm = 0.5 * rsinv * rbinv * (dmi * dmi + rs * rs + rb * rb);
            else
                xm = 0.5 * rsinv * rbinv * (dmi * dmi + rb * rb + rs * rs);
            (void)top_like;
            toroidal_eval(qc, xm, qm);
            if (with_image) {
                xp = 0.5 * rsinv * rbinv * (dpl * dpl + rs * rs + rb * rb);
                toroidal_eval(qc, xp, qp);
            }
            long p = (long)(jl - 2) + (long)nr * (kl - 2);
            for (int m = 0; m < mmax; ++m) {
                double v = with_image ? coef * (qp[m] + qm[m]) : coef * qm[m];
                c->green[((long)m * c->nb + b) * np + p] = v;
            }
        }
    }
}

static void green_build(orc_ctx *c) {
    const orc_grid *g = &c->g;
    qcoef_t qc;
    qcoef_init(&qc, g->isym, g->mmax);
    const int nr = c->nr, nz = c->nz;
    const int img = (g->isym != 1);
    const double zB = c->zhf_g[g->numz - 1];          /* tm.F90:101 */
    const double rB = c->rhf_g[g->numr - 1];          /* sm.F90:115 */
    const double rBinv = 1.0 / rB;
    const double zBot = c->zhf_g[0];                  /* bm.F90:101 */
    const int nrow = c->nb;
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nrow; ++b) {
        if (b < nr) {               /* top: jg = b+2 (tm) */
            int jg = b + 2;
            green_row(c, &qc, c->rhf_g[jg - 1], c->rhfinv_g[jg - 1], zB, 1, img, img ? 0 : 1, b);
        } else if (b < nr + nz) {   /* side: kg (sm) */
            int kg = b - nr + 2;
            green_row(c, &qc, rB, rBinv, c->zhf_g[kg - 1], 0, img, img ? 0 : 1, b);
        } else {                    /* bottom, isym 1 (bm) */
            int jg = b - nr - nz + 2;
            green_row(c, &qc, c->rhf_g[jg - 1], c->rhfinv_g[jg - 1], zBot, 1, 0, 1, b);
        }
    }
    qcoef_free(&qc);
}

/* Note on the side table: sm.F90 evaluates (zhf_g(kg) -+ zhf(kl)), i.e.
 * zb -+ z' with zb = zhf_g(kg); green_row uses the same differences. */

/* potsetup.F90:113-252: constants, bessel trig, ADI coefficients. */
static void coef_init(orc_ctx *c) {
    const orc_grid *g = &c->g;
    const int N = g->numphi, mmax = g->mmax;
    c->piinv = 1.0 / c->pi;
    c->four_pi = 4.0 * c->pi;
    c->factor = (g->isym == 3) ? -(2.0 * g->dr * c->dz * c->dphi) : -(g->dr * c->dz * c->dphi);
    double mi = 1.0;
    for (int M = 0; M < mmax; ++M) {
        double li = 1.0;
        for (int L = 0; L < N; ++L) {
            double arg = (g->isym == 3) ? c->dphi * (mi - 1.0) * (2.0 * li - 1.0)
                                        : 0.5 * c->dphi * (mi - 1.0) * (2.0 * li - 1.0);
            c->bes_cos[(long)M * N + L] = cos(arg);
            c->bes_sin[(long)M * N + L] = sin(arg);
            li = li + 1.0;
        }
        mi = mi + 1.0;
    }
    c->gamma = c->dzinv * c->dzinv;
    double drinv2 = c->drinv * c->drinv;
    double dphiinv2 = c->dphiinv * c->dphiinv;
    int lstop = N / 2 + 1;
    for (int L = 1; L <= N; ++L) {
        int mode;
        if (g->isym == 3)
            mode = (L <= lstop) ? (L - 1) * (L - 1) : (L - lstop) * (L - lstop);
        else
            mode = (L <= lstop) ? L - 1 : L - lstop;
        c->mode[L - 1] = mode;
        c->m1mode[L - 1] = (mode % 2 == 0) ? 1.0 : -1.0;
        c->elm[L - 1] = cos((double)mode * c->dphi);
    }
    const int numr = g->numr;
    for (int J = 2; J <= numr - 1; ++J) {
        c->alphar[J - 1] = -c->r_g[J] * c->rhfinv_g[J - 1] * drinv2;
        c->betar[J - 1] = -c->r_g[J - 1] * c->rhfinv_g[J - 1] * drinv2;
        c->alphaz[J - 1] = -c->r_g[J] * c->rhfinv_g[J - 1] * drinv2;
        c->betaz[J - 1] = -c->r_g[J - 1] * c->rhfinv_g[J - 1] * drinv2;
    }
    c->az = -c->gamma;
    c->cz = -c->gamma;
    for (int L = 0; L < N; ++L) {
        double em1 = c->elm[L] - 1.0;
        double *brb = c->brb + (long)L * numr;
        double *elz = c->elambdazb + (long)L * numr;
        for (int J = 3; J <= numr - 1; ++J)
            brb[J - 1] = 2.0 * drinv2 - 2.0 * em1 * dphiinv2 * c->rhfinv_g[J - 1] * c->rhfinv_g[J - 1];
        double az2 = 2.0 * em1 * dphiinv2 * c->rhfinv_g[1] * c->rhfinv_g[1];
        if (g->isym == 3)
            brb[1] = -c->alphar[1] - 2.0 * c->betar[1] - az2;
        else
            brb[1] = -c->alphar[1] + (c->m1mode[L] - 1.0) * c->betar[1] - az2;
        for (int J = 2; J <= numr - 1; ++J)
            elz[J - 1] = -2.0 * drinv2 + 2.0 * em1 * dphiinv2 * c->rhfinv_g[J - 1] * c->rhfinv_g[J - 1];
        if (g->isym == 3)
            elz[1] = c->alphaz[1] + 2.0 * c->betaz[1] + az2;
        else
            elz[1] = c->alphaz[1] - (c->m1mode[L] - 1.0) * c->betaz[1] + az2;
    }
    for (int K = 2; K <= g->numz - 1; ++K) c->bzb[K - 1] = 2.0 * c->gamma;
    if (g->isym != 1) c->bzb[1] = c->gamma;
}

int orc_setup(const orc_grid *gin, orc_ctx **out) {
    *out = NULL;
    if (!gin) { set_err("null grid"); return -1; }
    orc_grid g = *gin;
    if (g.numr < 5 || g.numz < 5) { set_err("numr and numz must be >= 5"); return -1; }
    if (!is_pow2(g.numphi) || g.numphi < 8) { set_err("numphi must be a power of two >= 8"); return -1; }
    if (g.isym < 1 || g.isym > 3) { set_err("isym must be 1, 2 or 3"); return -1; }
    if (g.mmax < 2 || g.mmax > 64 || g.mmax > g.numphi) { set_err("mmax out of range"); return -1; }
    if (!(g.dr > 0.0)) { set_err("dr must be positive"); return -1; }
    orc_ctx *c = calloc(1, sizeof *c);
    c->g = g;
    c->nr = g.numr - 2;
    c->nz = g.numz - 2;
    c->nb = (g.isym == 1) ? 2 * c->nr + c->nz : c->nr + c->nz;
    c->nplane = (long)g.numr * g.numz;
    c->ntot = c->nplane * g.numphi;
    c->r_g = calloc(g.numr, sizeof(double));
    c->rhf_g = calloc(g.numr, sizeof(double));
    c->rinv_g = calloc(g.numr, sizeof(double));
    c->rhfinv_g = calloc(g.numr, sizeof(double));
    c->zhf_g = calloc(g.numz, sizeof(double));
    c->bes_cos = calloc((size_t)g.mmax * g.numphi, sizeof(double));
    c->bes_sin = calloc((size_t)g.mmax * g.numphi, sizeof(double));
    c->mode = calloc(g.numphi, sizeof(int));
    c->elm = calloc(g.numphi, sizeof(double));
    c->m1mode = calloc(g.numphi, sizeof(double));
    c->alphar = calloc(g.numr, sizeof(double));
    c->betar = calloc(g.numr, sizeof(double));
    c->alphaz = calloc(g.numr, sizeof(double));
    c->betaz = calloc(g.numr, sizeof(double));
    c->brb = calloc((size_t)g.numphi * g.numr, sizeof(double));
    c->elambdazb = calloc((size_t)g.numphi * g.numr, sizeof(double));
    c->bzb = calloc(g.numz, sizeof(double));
    c->green = calloc((size_t)g.mmax * c->nb * c->nr * c->nz, sizeof(double));
    c->S = calloc((size_t)g.mmax * c->nb * 2, sizeof(double));
    c->potp = calloc((size_t)c->ntot, sizeof(double));
    c->rhop = calloc((size_t)c->ntot, sizeof(double));
    if (!c->green || !c->potp || !c->rhop) { orc_destroy(c); set_err("out of memory"); return -2; }
    grid_init(c);
    coef_init(c);
    green_build(c);
    *out = c;
    return 0;
}

void orc_destroy(orc_ctx *c) {
    if (!c) return;
    free(c->r_g); free(c->rhf_g); free(c->rinv_g); free(c->rhfinv_g); free(c->zhf_g);
    free(c->bes_cos); free(c->bes_sin); free(c->mode); free(c->elm); free(c->m1mode);
    free(c->alphar); free(c->betar); free(c->alphaz); free(c->betaz);
    free(c->brb); free(c->elambdazb); free(c->bzb);
    free(c->green); free(c->S); free(c->potp); free(c->rhop);
    free(c);
}

/* ------------------------------------------------------------------ */
/* Boundary potential (bessel.F90)                                     */
/* ------------------------------------------------------------------ */

/* bessel.F90:170-488 with identity reductions.  Reads the unzeroed rho over
 * J=2..numr-1, K=2..numz-1 and writes the Dirichlet planes of potp: top
 * K=numz, side J=numr and (isym 1) bottom K=1. */
static void bessel(orc_ctx *c, const double *rho) {
    const orc_grid *g = &c->g;
    const int numr = g->numr, numz = g->numz, N = g->numphi, mmax = g->mmax;
    const int nr = c->nr, nz = c->nz, nb = c->nb;
    const long np = (long)nr * nz;
    double *tmp = calloc((size_t)mmax * 2 * np, sizeof(double)); /* [m][cos|sin][p] */
    /* projections onto cos/sin(m phi_l), phi_l = (l - 1/2) dphi (bessel.F90:179-185, 267-274) */
#pragma omp parallel for
    for (long p = 0; p < np; ++p) {
        int J = (int)(p % nr) + 2, K = (int)(p / nr) + 2;
        double acc = 0.0;
        for (int L = 1; L <= N; ++L) acc = acc + rho[IX(c, J, K, L)];
        tmp[p] = acc;
        for (int m = 1; m < mmax; ++m) {
            double ac = 0.0, as = 0.0;
            const double *bc = c->bes_cos + (long)m * N, *bs = c->bes_sin + (long)m * N;
            for (int L = 1; L <= N; ++L) {
                double r = rho[IX(c, J, K, L)];
                ac = ac + r * bc[L - 1];
                as = as + r * bs[L - 1];
            }
            tmp[((long)m * 2 + 0) * np + p] = ac;
            tmp[((long)m * 2 + 1) * np + p] = as;
        }
    }
    /* contraction with the Green tables (bessel.F90:186-296) */
#pragma omp parallel for collapse(2)
    for (int m = 0; m < mmax; ++m) {
        for (int b = 0; b < nb; ++b) {
            const double *G = c->green + ((long)m * nb + b) * np;
            const double *tc = tmp + ((long)m * 2 + 0) * np, *ts = tmp + ((long)m * 2 + 1) * np;
            double sc = 0.0, ss = 0.0;
            for (long p = 0; p < np; ++p) {
                sc = sc + G[p] * tc[p];
                if (m > 0) ss = ss + G[p] * ts[p];
            }
            c->S[((long)m * nb + b) * 2 + 0] = sc;
            c->S[((long)m * nb + b) * 2 + 1] = ss;
        }
    }
    free(tmp);
    if (c->S_override) memcpy(c->S, c->S_override, sizeof(double) * (size_t)mmax * nb * 2);
    /* synthesis over m (bessel.F90:399-488) */
    double *line = malloc(sizeof(double) * (size_t)N);
    /* top, K = numz */
    for (int J = 2; J <= numr - 1; ++J) {
        int b = J - 2;
        for (int L = 0; L < N; ++L) line[L] = c->S[((long)0 * nb + b) * 2];
        for (int m = 1; m < mmax; ++m) {
            double sc = c->S[((long)m * nb + b) * 2], ss = c->S[((long)m * nb + b) * 2 + 1];
            for (int L = 0; L < N; ++L)
                line[L] = line[L] + 2.0 * (sc * c->bes_cos[(long)m * N + L]) + 2.0 * (ss * c->bes_sin[(long)m * N + L]);
        }
        for (int L = 1; L <= N; ++L) c->potp[IX(c, J, numz, L)] = c->factor * line[L - 1];
    }
    for (int L = 1; L <= N; ++L) {
        int Ls = (g->isym == 3) ? L : ((L <= N / 2) ? L + N / 2 : L - N / 2);
        c->potp[IX(c, 1, numz, L)] = c->potp[IX(c, 2, numz, Ls)];
        c->potp[IX(c, numr, numz, L)] = 0.0;
    }
    /* side, J = numr */
    for (int K = 2; K <= numz - 1; ++K) {
        int b = nr + K - 2;
        for (int L = 0; L < N; ++L) line[L] = c->S[((long)0 * nb + b) * 2];
        for (int m = 1; m < mmax; ++m) {
            double sc = c->S[((long)m * nb + b) * 2], ss = c->S[((long)m * nb + b) * 2 + 1];
            for (int L = 0; L < N; ++L)
                line[L] = line[L] + 2.0 * (sc * c->bes_cos[(long)m * N + L]) + 2.0 * (ss * c->bes_sin[(long)m * N + L]);
        }
        for (int L = 1; L <= N; ++L) c->potp[IX(c, numr, K, L)] = c->factor * line[L - 1];
    }
    for (int L = 1; L <= N; ++L) {
        c->potp[IX(c, numr, 1, L)] = (g->isym != 1) ? c->potp[IX(c, numr, 2, L)] : 0.0;
        c->potp[IX(c, numr, numz, L)] = 0.0;
    }
    /* bottom, K = 1 (isym 1) */
    if (g->isym == 1) {
        for (int J = 2; J <= numr - 1; ++J) {
            int b = nr + nz + J - 2;
            for (int L = 0; L < N; ++L) line[L] = c->S[((long)0 * nb + b) * 2];
            for (int m = 1; m < mmax; ++m) {
                double sc = c->S[((long)m * nb + b) * 2], ss = c->S[((long)m * nb + b) * 2 + 1];
                for (int L = 0; L < N; ++L)
                    line[L] = line[L] + 2.0 * (sc * c->bes_cos[(long)m * N + L]) + 2.0 * (ss * c->bes_sin[(long)m * N + L]);
            }
            for (int L = 1; L <= N; ++L) c->potp[IX(c, J, 1, L)] = c->factor * line[L - 1];
        }
        for (int L = 1; L <= N; ++L) {
            int Ls = (L <= N / 2) ? L + N / 2 : L - N / 2;
            c->potp[IX(c, 1, 1, L)] = c->potp[IX(c, 2, 1, Ls)];
            c->potp[IX(c, numr, 1, L)] = 0.0;
        }
    }
    free(line);
    (void)nz;
}

/* ------------------------------------------------------------------ */
/* ADI solve (helmadi.F90, tridagr.F90, tridagz.F90)                   */
/* ------------------------------------------------------------------ */

/* helmadi.F90:124-129 */
void orc_dt_schedule(const orc_ctx *c, int nsteps, double *dt) {
    const int numr = c->g.numr;
    dt[nsteps - 1] = 4.0 * (c->rinv_g[numr - 1] * c->rinv_g[numr - 1]);
    double alph = pow(c->r_g[numr - 1] * c->rinv_g[2], 2.0 / ((double)nsteps - 1.0));
    for (int I = 2; I <= nsteps; ++I) {
        int idx = nsteps + 1 - I;
        dt[idx - 1] = alph * dt[idx];
    }
}

/* Forward real FFT over phi of every (J,K) column and the slot reorder of
 * helmadi.F90:132-156: slot 1 = F_0, slot N/2+1 = F_{N/2},
 * slot L = Re F_{L-1} (L=2..N/2), slot L = -Im F_{L-N/2-1} (L>N/2+1). */
static void forward_slots(orc_ctx *c, double *a, double *ff) {
    const int N = c->g.numphi;
    const long np = c->nplane;
#pragma omp parallel
    {
        double *col = malloc(sizeof(double) * (size_t)N);
#pragma omp for
        for (long q = 0; q < np; ++q) {
            for (int L = 0; L < N; ++L) col[L] = a[q + np * L];
            orc_realft(col, 1, N, +1);
            ff[q] = col[0];
            ff[q + np * (N / 2)] = col[1];
            for (int L = 2; L <= N / 2; ++L) ff[q + np * (L - 1)] = col[2 * L - 2];
            for (int L = N / 2 + 2; L <= N; ++L) ff[q + np * (L - 1)] = -col[2 * (L - N / 2 - 1) + 1];
        }
        free(col);
    }
}

/* Un-reorder, inverse FFT and 2/N normalisation (helmadi.F90:357-392),
 * then the axis and equator conditions (helmadi.F90:396-411). */
static void inverse_slots(orc_ctx *c, const double *ff, double *a) {
    const orc_grid *g = &c->g;
    const int N = g->numphi, numr = g->numr, numz = g->numz;
    const long np = c->nplane;
    const double numphiinv = 1.0 / (double)N;
#pragma omp parallel
    {
        double *col = malloc(sizeof(double) * (size_t)N);
#pragma omp for
        for (long q = 0; q < np; ++q) {
            col[0] = ff[q];
            col[1] = ff[q + np * (N / 2)];
            for (int L = 2; L <= N / 2; ++L) col[2 * L - 2] = ff[q + np * (L - 1)];
            for (int L = N / 2 + 2; L <= N; ++L) col[2 * (L - N / 2 - 1) + 1] = -ff[q + np * (L - 1)];
            orc_realft(col, 1, N, -1);
            for (int L = 0; L < N; ++L) a[q + np * L] = 2.0 * numphiinv * col[L];
        }
        free(col);
    }
    if (g->isym == 3) {
        for (int L = 1; L <= N; ++L)
            for (int K = 1; K <= numz; ++K) a[IX(c, 1, K, L)] = a[IX(c, 2, K, L)];
    } else {
        for (int L = 1; L <= N / 2; ++L)
            for (int K = 1; K <= numz; ++K) {
                a[IX(c, 1, K, L)] = a[IX(c, 2, K, L + N / 2)];
                a[IX(c, 1, K, L + N / 2)] = a[IX(c, 2, K, L)];
            }
    }
    if (g->isym == 2 || g->isym == 3) {
        for (int L = 1; L <= N; ++L)
            for (int J = 1; J <= numr; ++J) a[IX(c, J, 1, L)] = a[IX(c, J, 2, L)];
    }
}

/* One Peaceman-Rachford step on one slot (helmadi.F90:197-353 with
 * tridagr.F90 and tridagz.F90).  fr = FFT of the zeroed density, fp = the
 * potential slot (updated in place), known/bet/gam are scratch. */
static void adi_step_slot(const orc_ctx *c, int L, double dtt, const double *fr, double *fp, double *known,
                          double *bet, double *gam) {
    const orc_grid *g = &c->g;
    const int numr = g->numr, numz = g->numz;
    const double gamma = c->gamma, four_pi = c->four_pi;
    const double *brb = c->brb + (long)(L - 1) * numr;
    const double *elz = c->elambdazb + (long)(L - 1) * numr;
#define P2(J, K) ((long)((J) - 1) + (long)numr * ((K) - 1))
    /* radial sweep */
    double dtm2g = dtt - 2.0 * gamma;
    for (int K = 2; K <= numz - 1; ++K) {
        for (int J = 2; J <= numr - 1; ++J) {
            double v;
            if (K == 2 && g->isym != 1)
                v = -(four_pi * fr[P2(J, K)]) + (dtt - gamma) * fp[P2(J, K)] + gamma * fp[P2(J, K + 1)];
            else
                v = -(four_pi * fr[P2(J, K)]) + dtm2g * fp[P2(J, K)] + gamma * (fp[P2(J, K + 1)] + fp[P2(J, K - 1)]);
            known[P2(J, K)] = v;
        }
        known[P2(numr - 1, K)] = known[P2(numr - 1, K)] - c->alphar[numr - 2] * fp[P2(numr, K)];
    }
    /* tridagr: ar = betar, cr = alphar, br = brb + dt */
    bet[1] = brb[1] + dtt;
    for (int J = 3; J <= numr - 1; ++J) {
        gam[J - 1] = c->alphar[J - 2] / bet[J - 2];
        bet[J - 1] = (brb[J - 1] + dtt) - c->betar[J - 1] * gam[J - 1];
    }
    for (int K = 2; K <= numz - 1; ++K) {
        fp[P2(2, K)] = known[P2(2, K)] / bet[1];
        for (int J = 3; J <= numr - 1; ++J)
            fp[P2(J, K)] = (known[P2(J, K)] - c->betar[J - 1] * fp[P2(J - 1, K)]) / bet[J - 1];
        for (int J = numr - 2; J >= 2; --J) fp[P2(J, K)] = fp[P2(J, K)] - gam[J] * fp[P2(J + 1, K)];
    }
    /* vertical sweep */
    for (int K = 2; K <= numz - 1; ++K) {
        for (int J = 2; J <= numr - 1; ++J) {
            double el = elz[J - 1] + dtt;
            double v = -(four_pi * fr[P2(J, K)]) + el * fp[P2(J, K)] - c->alphaz[J - 1] * fp[P2(J + 1, K)];
            if (J != 2) v = v - c->betaz[J - 1] * fp[P2(J - 1, K)];
            known[P2(J, K)] = v;
        }
    }
    for (int J = 2; J <= numr - 1; ++J)
        known[P2(J, numz - 1)] = known[P2(J, numz - 1)] + gamma * fp[P2(J, numz)];
    if (g->isym == 1)
        for (int J = 2; J <= numr - 1; ++J) known[P2(J, 2)] = known[P2(J, 2)] + gamma * fp[P2(J, 1)];
    /* tridagz: az = cz = -gamma, bz = bzb + dt */
    bet[1] = c->bzb[1] + dtt;
    for (int K = 3; K <= numz - 1; ++K) {
        gam[K - 1] = c->cz / bet[K - 2];
        bet[K - 1] = (c->bzb[K - 1] + dtt) - c->az * gam[K - 1];
    }
    for (int J = 2; J <= numr - 1; ++J) fp[P2(J, 2)] = known[P2(J, 2)] / bet[1];
    for (int K = 3; K <= numz - 1; ++K)
        for (int J = 2; J <= numr - 1; ++J)
            fp[P2(J, K)] = (known[P2(J, K)] - c->az * fp[P2(J, K - 1)]) / bet[K - 1];
    for (int K = numz - 2; K >= 2; --K)
        for (int J = 2; J <= numr - 1; ++J) fp[P2(J, K)] = fp[P2(J, K)] - gam[K] * fp[P2(J, K + 1)];
#undef P2
}

static void adi_cycle(orc_ctx *c, const double *dt, int nsteps, const double *ffr, double *ffp) {
    const int N = c->g.numphi;
    const long np = c->nplane;
    const int nmax = (c->g.numr > c->g.numz) ? c->g.numr : c->g.numz;
#pragma omp parallel
    {
        double *known = calloc((size_t)np, sizeof(double));
        double *bet = calloc((size_t)nmax, sizeof(double));
        double *gam = calloc((size_t)nmax, sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int L = 1; L <= N; ++L)
            for (int I = 0; I < nsteps; ++I)
                adi_step_slot(c, L, dt[I], ffr + np * (L - 1), ffp + np * (L - 1), known, bet, gam);
        free(known);
        free(bet);
        free(gam);
    }
}

/* Weighted slot-space relative residual ||-4 pi rho_hat - A phi_hat|| /
 * ||4 pi rho_hat|| over the interior, with Parseval weights 1 (slots 1 and
 * N/2+1) and 2 (others) so that it equals the physical-space L2 ratio. */
static double slot_residual(const orc_ctx *c, const double *ffr, const double *ffp) {
    const orc_grid *g = &c->g;
    const int numr = g->numr, numz = g->numz, N = g->numphi;
    const long np = c->nplane;
    double num = 0.0, den = 0.0;
#pragma omp parallel for reduction(+ : num, den)
    for (int L = 1; L <= N; ++L) {
        const double *fr = ffr + np * (L - 1), *fp = ffp + np * (L - 1);
        const double *brb = c->brb + (long)(L - 1) * numr;
        double w = (L == 1 || L == N / 2 + 1) ? 1.0 : 2.0;
        double sn = 0.0, sd = 0.0;
        for (int K = 2; K <= numz - 1; ++K)
            for (int J = 2; J <= numr - 1; ++J) {
                long q = (J - 1) + (long)numr * (K - 1);
                double ar = brb[J - 1] * fp[q] + c->alphar[J - 1] * fp[q + 1];
                if (J > 2) ar += c->betar[J - 1] * fp[q - 1];
                double az = c->bzb[K - 1] * fp[q] - c->gamma * fp[q + numr];
                if (K > 2 || g->isym == 1) az -= c->gamma * fp[q - numr];
                double b = -c->four_pi * fr[q];
                double r = b - ar - az;
                sn += r * r;
                sd += b * b;
            }
        num += w * sn;
        den += w * sd;
    }
    return den > 0.0 ? sqrt(num / den) : sqrt(num);
}

/* Weighted relative change ||phi_hat - prev|| / ||phi_hat|| over the
 * interior: the stop test of the converged form.  The normwise residual
 * above has an FP64 floor (~6e-11 at 66x66x64, from near-axis azimuthal
 * coefficients of order 1/(rhf dphi)^2) while the potential itself
 * converges to ~1e-14, so the iteration stops on the update. */
static double slot_update(const orc_ctx *c, const double *prev, const double *ffp) {
    const orc_grid *g = &c->g;
    const int numr = g->numr, numz = g->numz, N = g->numphi;
    const long np = c->nplane;
    double num = 0.0, den = 0.0;
#pragma omp parallel for reduction(+ : num, den)
    for (int L = 1; L <= N; ++L) {
        double w = (L == 1 || L == N / 2 + 1) ? 1.0 : 2.0, sn = 0.0, sd = 0.0;
        for (int K = 2; K <= numz - 1; ++K)
            for (int J = 2; J <= numr - 1; ++J) {
                long q = np * (L - 1) + (J - 1) + (long)numr * (K - 1);
                double d = ffp[q] - prev[q];
                sn += d * d;
                sd += ffp[q] * ffp[q];
            }
        num += w * sn;
        den += w * sd;
    }
    return den > 0.0 ? sqrt(num / den) : sqrt(num);
}

static void zero_rhop(orc_ctx *c, const double *rho) {
    const orc_grid *g = &c->g;
    const int numr = g->numr, numz = g->numz, N = g->numphi;
    memcpy(c->rhop, rho, sizeof(double) * (size_t)c->ntot);
    for (int L = 1; L <= N; ++L) {
        for (int J = 1; J <= numr; ++J) {
            c->rhop[IX(c, J, numz - 1, L)] = 0.0;
            c->rhop[IX(c, J, numz, L)] = 0.0;
            if (g->isym == 1) {
                c->rhop[IX(c, J, 1, L)] = 0.0;
                c->rhop[IX(c, J, 2, L)] = 0.0;
            }
        }
        for (int K = 1; K <= numz; ++K) {
            c->rhop[IX(c, numr - 1, K, L)] = 0.0;
            c->rhop[IX(c, numr, K, L)] = 0.0;
        }
    }
}

/* helmadi.F90:6-417 (and the converged variant when max_cycles > 1). */
static int helmadi(orc_ctx *c, int nsteps, int converged, double tol, int max_cycles, int *cycles_out,
                   double *resid_out) {
    const long ntot = c->ntot;
    double *dt = malloc(sizeof(double) * (size_t)nsteps);
    double *ffr = malloc(sizeof(double) * (size_t)ntot);
    double *ffp = malloc(sizeof(double) * (size_t)ntot);
    if (!dt || !ffr || !ffp) { free(dt); free(ffr); free(ffp); set_err("out of memory"); return -2; }
    orc_dt_schedule(c, nsteps, dt);
    forward_slots(c, c->rhop, ffr);
    forward_slots(c, c->potp, ffp);
    int cyc = 0;
    double *prev = converged ? malloc(sizeof(double) * (size_t)ntot) : NULL;
    for (;;) {
        if (prev) memcpy(prev, ffp, sizeof(double) * (size_t)ntot);
        adi_cycle(c, dt, nsteps, ffr, ffp);
        ++cyc;
        if (!converged) break;
        if (slot_update(c, prev, ffp) <= tol || cyc >= max_cycles) break;
    }
    free(prev);
    if (resid_out) *resid_out = slot_residual(c, ffr, ffp);
    if (cycles_out) *cycles_out = cyc;
    inverse_slots(c, ffp, c->potp);
    free(dt);
    free(ffr);
    free(ffp);
    return 0;
}

/* potential_solver.F90:6-109 with explicit step control. */
static int solve_common(orc_ctx *c, const double *rho, double *pot, int nsteps, int cold, int converged,
                        double tol, int max_cycles, int *cycles_out, double *resid_out) {
    if (!c || !rho || !pot) { set_err("null argument"); return -1; }
    if (nsteps < 1) { set_err("nsteps must be >= 1"); return -1; }
    for (long i = 0; i < c->ntot; ++i)
        if (!isfinite(rho[i])) { set_err("non-finite density"); return -3; }
    zero_rhop(c, rho);
    if (cold) memset(c->potp, 0, sizeof(double) * (size_t)c->ntot);
    bessel(c, rho);
    int rc = helmadi(c, nsteps, converged, tol, max_cycles, cycles_out, resid_out);
    if (rc) return rc;
    memcpy(pot, c->potp, sizeof(double) * (size_t)c->ntot);
    return 0;
}

int orc_potential_solver(orc_ctx *c, const double *rho, double *pot, int tstep) {
    int warm = tstep > 1;
    return solve_common(c, rho, pot, warm ? 5 : 20, !warm, 0, 0.0, 1, NULL, NULL);
}

int orc_solve_nsteps(orc_ctx *c, const double *rho, double *pot, int nsteps, int cold) {
    return solve_common(c, rho, pot, nsteps, cold, 0, 0.0, 1, NULL, NULL);
}

int orc_solve_converged(orc_ctx *c, const double *rho, double *pot, int nsteps, int cold, double tol,
                        int max_cycles, int *cycles_out, double *resid_out) {
    if (max_cycles < 1) max_cycles = 1;
    return solve_common(c, rho, pot, nsteps, cold, 1, tol, max_cycles, cycles_out, resid_out);
}

/* Test hook (not part of the reference algorithm): later solves use the
 * given boundary moments S[m][b][cos|sin] in place of the contraction's,
 * so that a test can measure how an error in S moves the potential.  NULL
 * restores the contraction.  The array must outlive the solves. */
void orc_set_moments_override(orc_ctx *c, const double *S) { c->S_override = S; }

/* Replaces the kept potential potp (COMMON /potarrays/) with pot, as a
 * continuation restart that restored potp would. */
void orc_set_potential(orc_ctx *c, const double *pot) {
    memcpy(c->potp, pot, sizeof(double) * (size_t)c->ntot);
}

double orc_residual(orc_ctx *c, const double *rho, const double *pot) {
    const long ntot = c->ntot;
    double *ffr = malloc(sizeof(double) * (size_t)ntot);
    double *ffp = malloc(sizeof(double) * (size_t)ntot);
    double *tmp = malloc(sizeof(double) * (size_t)ntot);
    zero_rhop(c, rho);
    memcpy(tmp, pot, sizeof(double) * (size_t)ntot);
    forward_slots(c, c->rhop, ffr);
    forward_slots(c, tmp, ffp);
    double r = slot_residual(c, ffr, ffp);
    free(ffr);
    free(ffp);
    free(tmp);
    return r;
}
