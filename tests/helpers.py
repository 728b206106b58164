"""Shared helpers of the test suite (density fields and error norms)."""
import numpy as np


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def smooth_density(numr, numz, numphi, dr, isym=2, seed=7):
    """A smooth, non-axisymmetric density with seeded noise for small grids."""
    from bipoly_hydro_b200 import fields

    x, y, z = fields.coordinates(numr, numz, numphi, dr, isym)
    R = (numr - 2) * dr
    rho = np.exp(-((x - 0.35 * R) ** 2 + (y + 0.1 * R) ** 2 + z ** 2) / (0.25 * R) ** 2)
    rho += 0.6 * np.exp(-((x + 0.4 * R) ** 2 + y ** 2 + (z - 0.05 * R) ** 2) / (0.2 * R) ** 2)
    rng = np.random.Generator(np.random.PCG64(seed))
    rho *= 1.0 + 1e-3 * rng.uniform(-1.0, 1.0, size=rho.shape)
    return np.asfortranarray(rho + 1e-10)
