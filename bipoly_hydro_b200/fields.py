"""Seeded synthetic density fields of the benchmark grids.

The reference's models come from its SCF code as files on disk (scfin,
scfin_frac.F90:105-125); none ship with it, so the benchmark workloads use
analytic polytrope pairs of the stated shapes, sizes and value ranges.  Grid
zone (J, K, L) sits at cylindrical (rhf_g(J), zhf_g(K), phi = (L-1) dphi)
(setup_frac.F90:374-463), with z >= 0 for isym 2/3 and z centred for isym 1.
Arrays are Fortran-ordered (numr, numz, numphi) float64.
"""
from __future__ import annotations

import numpy as np

DEFAULT_SEED = 20261203


def coordinates(numr: int, numz: int, numphi: int, dr: float, isym: int = 2):
    """Cartesian (x, y, z) of every zone centre, each (numr, numz, numphi)."""
    J = np.arange(1, numr + 1, dtype=np.float64)
    K = np.arange(1, numz + 1, dtype=np.float64)
    L = np.arange(1, numphi + 1, dtype=np.float64)
    r = (J - 2.0) * dr + 0.5 * dr
    if isym != 1:
        z = (K - 1.5) * dr
    else:
        z = -(numz // 2) * dr + (K - 0.5) * dr
    phi = (L - 1.0) * (2.0 * np.pi / numphi)
    R3, Z3, P3 = np.meshgrid(r, z, phi, indexing="ij")
    return R3 * np.cos(P3), R3 * np.sin(P3), Z3


def _lane_emden_n1(s: np.ndarray, radius: float) -> np.ndarray:
    """n = 1 polytrope profile sin(pi s/R)/(pi s/R) inside R, 0 outside."""
    u = np.pi * s / radius
    with np.errstate(invalid="ignore", divide="ignore"):
        prof = np.where(u > 0, np.sin(u) / np.where(u > 0, u, 1.0), 1.0)
    return np.where(s < radius, prof, 0.0)


def two_polytropes(numr=66, numz=66, numphi=64, dr=1.0 / 62.0, isym=2, seed=DEFAULT_SEED,
                   radius=0.25, centre_r=0.4, rho_c=(1.0, 0.7), floor=1e-10, noise=1e-3):
    """Two n=1 polytropes at (r=0.4, phi=0) and (r=0.4, phi=pi) on z=0, floor and seeded noise."""
    x, y, z = coordinates(numr, numz, numphi, dr, isym)
    rho = np.zeros_like(x)
    for rc, ang in zip(rho_c, (0.0, np.pi)):
        cx, cy = centre_r * np.cos(ang), centre_r * np.sin(ang)
        s = np.sqrt((x - cx) ** 2 + (y - cy) ** 2 + z ** 2)
        rho += rc * _lane_emden_n1(s, radius)
    rho = np.maximum(rho, floor)
    rng = np.random.Generator(np.random.PCG64(seed))
    rho *= 1.0 + noise * rng.uniform(-1.0, 1.0, size=rho.shape)
    return np.asfortranarray(rho)


def bipolytrope_pair(numr=130, numz=98, numphi=256, dr=1.0 / 126.0, isym=2, seed=DEFAULT_SEED,
                     r1=0.3, r2=0.22, separation=0.9, mass_ratio=0.5, core_jump=2.0, core_frac=0.4,
                     floor=1e-10, noise=0.0):
    """Binary of two bipolytropes on the x-axis about the centre of mass.

    Each star is an n=1 profile with the density multiplied by ``core_jump``
    inside ``core_frac`` of its radius; the secondary's central density is set
    so that the grid mass ratio M2/M1 equals ``mass_ratio``.
    """
    x, y, z = coordinates(numr, numz, numphi, dr, isym)
    q, a = mass_ratio, separation
    x1, x2 = a * q / (1.0 + q), -a / (1.0 + q)

    def star(cx, radius):
        s = np.sqrt((x - cx) ** 2 + y ** 2 + z ** 2)
        prof = _lane_emden_n1(s, radius)
        return prof * np.where(s < core_frac * radius, core_jump, 1.0)

    s1, s2 = star(x1, r1), star(x2, r2)
    # zone volume ~ rhf: the mass ratio is a ratio of sum(rho * rhf)
    rhf = np.sqrt(x ** 2 + y ** 2)
    m1, m2 = float((s1 * rhf).sum()), float((s2 * rhf).sum())
    rho = s1 + (q * m1 / m2) * s2
    rho = np.maximum(rho, floor)
    if noise:
        rng = np.random.Generator(np.random.PCG64(seed))
        rho *= 1.0 + noise * rng.uniform(-1.0, 1.0, size=rho.shape)
    return np.asfortranarray(rho)


def rotate(rho: np.ndarray, slots: int = 1) -> np.ndarray:
    """Rigid rotation by slots * dphi (one azimuthal zone per time step)."""
    return np.asfortranarray(np.roll(rho, slots, axis=2))
