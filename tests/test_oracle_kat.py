"""Known-answer tests that pin the CPU oracle (no GPU).

The reference has no tests or golden vectors and cannot be compiled here, so
the oracle's restatement is pinned against independent mathematics: special
functions against mpmath/scipy, the azimuthal FFT against numpy, single-mode
densities, a spherically symmetric density with a closed-form potential, the
converged discrete system, and the committed golden fixtures.
"""
import math
import os

import numpy as np
import pytest

from tests.helpers import rel_l2, smooth_density

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# ---------------------------------------------------------------- special functions
@pytest.mark.parametrize("x", [0.25, 0.5, 1.0, 1.5, 3.7, 10.25, 30.5, 60.75, 111.0, 140.5])
def test_gammln_is_lanczos_accurate(oracle_mod, x):
    """gammln.F90's 6-term Lanczos form: within its published ~2e-10 bound of ln Gamma."""
    assert abs(oracle_mod.gammln(x) - math.lgamma(x)) <= 2e-10 * max(1.0, abs(math.lgamma(x)))


def test_gammln_is_not_exact_lgamma(oracle_mod):
    """Parity trap: the tables need the approximation, which differs from lgamma."""
    assert abs(oracle_mod.gammln(111.0) - math.lgamma(111.0)) > 1e-12


@pytest.mark.parametrize("y", [1e-6, 0.01, 0.3, 0.7, 0.99, 1.0, 2.5])
def test_carlson_rf_rd(oracle_mod, y):
    import scipy.special as sp

    assert oracle_mod.rf(0.0, y, 1.0) == pytest.approx(sp.elliprf(0.0, y, 1.0), rel=2e-15)
    assert oracle_mod.rd(0.0, y, 1.0) == pytest.approx(sp.elliprd(0.0, y, 1.0), rel=2e-15)
    assert oracle_mod.rf(0.3, y, 2.0) == pytest.approx(sp.elliprf(0.3, y, 2.0), rel=2e-15)


def test_carlson_invalid_arguments_are_nan(oracle_mod):
    assert math.isnan(oracle_mod.rf(-1.0, 1.0, 1.0))
    assert math.isnan(oracle_mod.rd(0.0, 0.0, 1.0))


@pytest.mark.parametrize("k", [0.05, 0.3, 0.6, 0.9, 0.99, 0.9999])
def test_complete_elliptic_integrals(oracle_mod, k):
    import scipy.special as sp

    assert oracle_mod.ellf(k) == pytest.approx(sp.ellipk(k * k), rel=3e-15)
    assert oracle_mod.elle(k) == pytest.approx(sp.ellipe(k * k), rel=3e-15)


def _legenq(m, x):
    import mpmath

    mpmath.mp.dps = 40
    return float(mpmath.re(mpmath.legenq(m - 0.5, 0, x, type=3)))


@pytest.mark.parametrize("x", [1.0005, 1.005, 1.02])
def test_toroidal_elliptic_branch(oracle_mod, x):
    """x < 1.025: K/E plus upward recurrence (tm.F90:215-225)."""
    q = oracle_mod.toroidal(x, 2, 30)
    for m in range(30):
        ref = _legenq(m, x)
        tol = 2e-12 if m < 10 else 5e-10   # cancellation in x mu K - lambda E, then upward recurrence
        assert abs(q[m] - ref) <= tol * abs(ref), (m, q[m], ref)


@pytest.mark.parametrize("x", [1.5, 3.0, 20.0])
def test_toroidal_series_branch(oracle_mod, x):
    """x >= 1.025 far from the cutoff: the 111-term series (tm.F90:226-240) converges."""
    q = oracle_mod.toroidal(x, 2, 30)
    for m in range(30):
        ref = _legenq(m, x)
        assert abs(q[m] - ref) <= 1e-11 * abs(ref), (m, q[m], ref)


def test_toroidal_series_truncation_near_cutoff_is_the_references(oracle_mod):
    """Just above 1.025 the reference's 111 terms are too few: the oracle must
    reproduce the truncated sum (evaluated independently in mpmath with the
    same 111 terms), not the exact Q."""
    import mpmath

    mpmath.mp.dps = 40
    x = mpmath.mpf("1.03")
    q = oracle_mod.toroidal(1.03, 2, 30)
    for m in (0, 5, 29):
        aa, bb, cc = (m + 1.5) / 2, (m + 0.5) / 2, m + 1
        pref = mpmath.sqrt(mpmath.pi) * mpmath.gamma(m + 0.5) / mpmath.gamma(m + 1) / (2 * x) ** (m + 0.5)
        terms = sum(mpmath.rf(aa, n) * mpmath.rf(bb, n) / (mpmath.rf(cc, n) * mpmath.factorial(n)) * x ** (-2 * n)
                    for n in range(111))
        truncated = float(pref * terms)
        assert abs(q[m] - truncated) <= 1e-9 * abs(truncated), m   # Lanczos gammln ~1e-10
    assert abs(q[29] - _legenq(29, 1.03)) > 1e-3 * abs(q[29])      # and it is not the exact Q


# ---------------------------------------------------------------- azimuthal FFT
@pytest.mark.parametrize("n", [16, 64, 256, 512])
def test_realft_is_plus_i_dft(oracle_mod, n):
    f = np.random.default_rng(n).standard_normal(n)
    d = oracle_mod.realft(f, +1)
    F = np.conj(np.fft.rfft(f))  # sum f_l exp(+2 pi i k l / n)
    ref = np.empty(n)
    ref[0], ref[1] = F[0].real, F[n // 2].real
    ref[2::2], ref[3::2] = F[1:n // 2].real, F[1:n // 2].imag
    assert np.abs(d - ref).max() <= 1e-14 * np.abs(ref).max()
    back = oracle_mod.realft(d, -1) * 2.0 / n
    assert np.abs(back - f).max() <= 1e-14 * np.abs(f).max()


# ---------------------------------------------------------------- solver structure
def test_dt_schedule_is_geometric(oracle_mod):
    o = oracle_mod.Oracle(34, 26, 16, 1.0 / 30.0, 2, 6)
    for n in (5, 20):
        dt = o.dt_schedule(n)
        r_numr, r3 = 32.0 / 30.0, 1.0 / 30.0
        assert dt[-1] == pytest.approx(4.0 / r_numr ** 2, rel=1e-15)
        assert dt[0] == pytest.approx(4.0 / r3 ** 2, rel=1e-12)
        ratios = dt[:-1] / dt[1:]
        assert np.allclose(ratios, ratios[0], rtol=1e-13)
    o.close()


@pytest.mark.parametrize("isym", [1, 2, 3])
def test_slot_modes(oracle_mod, isym):
    o = oracle_mod.Oracle(14, 12, 32, 0.1, isym, 6)
    modes = o.slot_modes()
    lin = np.r_[np.arange(17), np.arange(1, 16)]
    assert np.array_equal(modes, lin ** 2 if isym == 3 else lin)  # potsetup.F90:157-170 (isym 3 squares)
    o.close()


@pytest.mark.parametrize("m", [0, 2, 5])
def test_single_mode_density_gives_single_mode_potential(oracle_mod, m):
    """rho = f(r,z) cos(m phi + c): the interior potential has only azimuthal mode m."""
    numr, numz, numphi, dr = 34, 26, 32, 1.0 / 30.0
    o = oracle_mod.Oracle(numr, numz, numphi, dr, 2, 12)
    from bipoly_hydro_b200 import fields

    x, y, z = fields.coordinates(numr, numz, numphi, dr, 2)
    r, phi = np.hypot(x, y), np.arctan2(y, x)
    rho = np.asfortranarray(np.exp(-((r - 0.4) ** 2 + z ** 2) / 0.02) * (1.5 + np.cos(m * phi + 0.3)) if m == 0
                            else np.exp(-((r - 0.4) ** 2 + z ** 2) / 0.02) * np.cos(m * phi + 0.3))
    pot, _, _ = o.solve_converged(rho, 20, True, 1e-13, 50)
    spec = np.abs(np.fft.rfft(pot[2:-1, 2:-1, :], axis=2))
    total = spec.max()
    others = np.delete(spec, m, axis=2)
    assert others.max() <= 1e-11 * total
    o.close()


def test_gaussian_sphere_converges_to_closed_form(oracle_mod):
    """A spherical Gaussian at the origin has Phi = -M erf(s / (sqrt2 sigma)) / s
    (G = 1).  The converged discrete solution must approach it at second order."""
    from scipy.special import erf

    from bipoly_hydro_b200 import fields

    sigma = 0.12
    errs = []
    for numr, numphi in ((34, 16), (66, 16)):
        dr = 1.0 / (numr - 4)
        o = oracle_mod.Oracle(numr, numr, numphi, dr, 2, 8)
        x, y, z = fields.coordinates(numr, numr, numphi, dr, 2)
        s = np.sqrt(x ** 2 + y ** 2 + z ** 2)
        rho = np.asfortranarray(np.exp(-0.5 * (s / sigma) ** 2))
        mass = (2 * np.pi * sigma ** 2) ** 1.5
        exact = -mass * erf(s / (np.sqrt(2) * sigma)) / s
        pot, _, _ = o.solve_converged(rho, 20, True, 1e-13, 50)
        sl = (slice(1, -1), slice(1, -1), slice(None))
        errs.append(rel_l2(pot[sl], exact[sl]))
        o.close()
    assert errs[0] < 5e-3
    assert errs[1] < 0.35 * errs[0]      # ~4x per halving of dr


def test_converged_solution_is_schedule_independent(oracle_mod):
    grid = (34, 26, 32, 1.0 / 30.0, 2, 12)
    o = oracle_mod.Oracle(*grid)
    rho = smooth_density(*grid[:5])
    p20, c20, r20 = o.solve_converged(rho, 20, True, 1e-13, 100)
    p5, c5, r5 = o.solve_converged(rho, 5, True, 1e-13, 400)
    assert rel_l2(p5, p20) <= 1e-12
    assert r20 <= 1e-9 and r5 <= 1e-9          # the FP64 residual floor is ~1e-11 here
    assert c20 < c5
    o.close()


def test_warm_start_is_closer_than_cold(oracle_mod):
    """potential_solver: 5 warm steps from the previous solution beat 5 cold steps."""
    grid = (34, 26, 32, 1.0 / 30.0, 2, 12)
    o = oracle_mod.Oracle(*grid)
    rho = smooth_density(*grid[:5])
    conv, _, _ = o.solve_converged(rho, 20, True, 1e-13, 100)
    o.potential_solver(rho, 0)
    warm = o.potential_solver(rho, 2)
    cold5 = o.solve_nsteps(rho, 5, True)
    assert rel_l2(warm, conv) < 0.1 * rel_l2(cold5, conv)
    o.close()


# ---------------------------------------------------------------- golden fixtures
GOLDEN_FILES = sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.mark.parametrize("name", GOLDEN_FILES)
def test_oracle_reproduces_golden_fixture(oracle_mod, name):
    g = np.load(os.path.join(GOLDEN, name))
    numr, numz, numphi, isym, mmax = (int(v) for v in g["grid"])
    o = oracle_mod.Oracle(numr, numz, numphi, float(g["dr"]), isym, mmax)
    rho = np.asfortranarray(g["rho"])
    assert rel_l2(o.potential_solver(rho, 0), g["cold"]) <= 1e-14
    warm = o.potential_solver(np.asfortranarray(np.roll(rho, 1, axis=2)), 2)
    assert rel_l2(warm, g["warm"]) <= 1e-14
    assert rel_l2(o.moments_S(), g["S_warm"]) <= 1e-14
    G = o.green()
    assert rel_l2(G[0, :4], g["green_m0"]) <= 1e-15
    assert rel_l2(G[-1, :4], g["green_mlast"]) <= 1e-15
    o.close()
