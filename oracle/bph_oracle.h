/*
 * bph_oracle.h -- CPU restatement of bipoly_hydro's self-gravity Poisson
 * solve, for one MPI rank, in plain C (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA solver in bipoly_hydro_b200/ and the timed CPU baseline in
 * bench.py.  The product path never links, loads or calls it.
 *
 * Parity status: UNPINNED by the reference itself.  The reference is
 * Fortran 90 + MPI with no tests, no golden vectors and no fixtures, and
 * no Fortran compiler exists in this image, so it cannot be run to pin
 * this restatement.  The restatement is pinned instead against analytic
 * known answers (mpmath toroidal functions, scipy elliptic integrals, a
 * direct DFT, dense tridiagonal solves, a uniform-sphere potential and a
 * converged discrete residual) in tests/test_oracle_*.py.
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef BPH_ORACLE_H
#define BPH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid {
    int numr;      /* radial zones incl. guard J=1 and boundary J=numr (runhydro.h:1) */
    int numz;      /* vertical zones incl. guard K=1 and boundary K=numz (runhydro.h:2) */
    int numphi;    /* azimuthal zones, power of two (runhydro.h:3) */
    double dr;     /* radial spacing; dz = dr (setup_frac.F90:374-375) */
    int isym;      /* 1 none, 2 equatorial, 3 pi+equatorial (setup_frac.F90:182-270) */
    int mmax;      /* boundary-solve azimuthal modes, 30 in pot.h:3 */
} orc_grid;

typedef struct orc_ctx orc_ctx;

/* potsetup.F90:6 + tm/sm/bm: build grid, trig tables, Green tables, ADI
 * coefficients.  Returns 0 or a negative error code. */
int orc_setup(const orc_grid *g, orc_ctx **out);
void orc_destroy(orc_ctx *c);

/* potential_solver.F90:6-109: rho, pot are (numr,numz,numphi) column-major.
 * tstep > 1 selects a warm start (5 ADI steps from the previous potp),
 * otherwise cold (20 steps from potp = 0). */
int orc_potential_solver(orc_ctx *c, const double *rho, double *pot, int tstep);

/* Same driver with an explicit ADI step count; cold != 0 zeroes potp. */
int orc_solve_nsteps(orc_ctx *c, const double *rho, double *pot, int nsteps, int cold);

/* Converged form: the nsteps schedule is repeated in Fourier-slot space
 * until the weighted relative change of phi_hat over one cycle is <= tol
 * or max_cycles cycles ran; resid_out gets the weighted relative residual
 * ||-4 pi rho_hat - A phi_hat|| / ||4 pi rho_hat|| of the result. */
int orc_solve_converged(orc_ctx *c, const double *rho, double *pot, int nsteps,
                        int cold, double tol, int max_cycles,
                        int *cycles_out, double *resid_out);

/* Sets the kept potential potp (warm-start state) to pot. */
void orc_set_potential(orc_ctx *c, const double *pot);
/* Test hook: boundary moments S[m][b][2] used by later solves instead of the
 * contraction's (NULL: the contraction again). */
void orc_set_moments_override(orc_ctx *c, const double *S);

/* Relative residual of a physical-space potential (after a solve) in slot
 * space, the same measure orc_solve_converged uses. */
double orc_residual(orc_ctx *c, const double *rho, const double *pot);

/* Accessors for tests. */
int orc_num_boundary_rows(const orc_ctx *c);
/* Green tables in layout G[m][b][p], p = (jl-2) + (numr-2)*(kl-2),
 * b = top jg-2 | side (numr-2)+kg-2 | bottom (isym=1). */
const double *orc_green(const orc_ctx *c);
/* Boundary moments S[m][b][2] (cos, sin) of the last bessel call. */
const double *orc_moments_S(const orc_ctx *c);
/* ADI pseudo-timestep schedule (helmadi.F90:124-129). */
void orc_dt_schedule(const orc_ctx *c, int nsteps, double *dt);
/* Per-slot mode number (potsetup.F90:157-173). */
int orc_slot_mode(const orc_ctx *c, int slot0);

/* Special functions (published methods; see the .c file). */
double orc_gammln(double x);
double orc_rf(double x, double y, double z);
double orc_rd(double x, double y, double z);
double orc_ellf(double k);
double orc_elle(double k);
/* Toroidal functions Q_{m-1/2}(x) (isym 1,2) or the even-degree set
 * (isym 3) for m = 0..mmax-1, the way tm.F90:118-193 evaluates them. */
void orc_toroidal(double x, int isym, int mmax, double *q);

/* realft.F90:5-77 on one strided column of n reals (n power of two). */
void orc_realft(double *data, long stride, int n, int isign);

/* Number of OpenMP threads the oracle uses (1 without OpenMP). */
int orc_num_threads(void);
void orc_set_num_threads(int n);

/* Error text for the last failing call. */
const char *orc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
