"""bph_scf_step: one SCF-like iteration on the device (density update with a
seeded perturbation, renormalisation to a fixed mass, potential_solver),
against a numpy restatement of the update and the oracle's solve of the
updated density."""
import numpy as np
import pytest

from tests.helpers import rel_l2, smooth_density

pytestmark = pytest.mark.gpu

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def scf_normal(seed, iteration, n):
    """xi of zones 0..n-1 (Fortran order), the generator bph_scf_step documents."""
    with np.errstate(over="ignore"):
        key = np.uint64(seed) ^ (np.uint64(0xD1B54A32D192ED03) * np.uint64(iteration + 1))
        i = np.arange(1, n + 1, dtype=np.uint64)
        z = _splitmix64(key + np.uint64(0x9E3779B97F4A7C15) * i)
    u1 = ((z >> np.uint64(32)).astype(np.float64) + 0.5) * (1.0 / 4294967296.0)
    u2 = ((z & np.uint64(0xFFFFFFFF)).astype(np.float64) + 0.5) * (1.0 / 4294967296.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)


def interior_mass(rho, dr, numphi):
    numr = rho.shape[0]
    rhf = (np.arange(numr) - 0.5) * dr
    return float((rho[1:-1, 1:-1, :] * rhf[1:-1, None, None]).sum()) * dr * dr * (2.0 * np.pi / numphi)


def scf_update(rho, eps, mass, seed, iteration, dr):
    numphi = rho.shape[2]
    xi = scf_normal(seed, iteration, rho.size).reshape(rho.shape, order="F")
    before = interior_mass(rho, dr, numphi)
    rn = 0.9 * rho + 0.1 * (rho * (1.0 + eps * xi))
    target = mass if mass > 0 else before
    return np.asfortranarray(rn * (target / interior_mass(rn, dr, numphi))), target


def test_normal_deviates_look_normal():
    xi = scf_normal(20261203, 4, 200000)
    assert abs(xi.mean()) < 0.01 and abs(xi.std() - 1.0) < 0.01


def test_scf_sequence_matches_update_and_oracle(bph, oracle_mod):
    import torch

    grid = (34, 26, 64, 1.0 / 30.0, 2, 30)
    numr, numz, numphi, dr, isym, _ = grid
    rho = smooth_density(numr, numz, numphi, dr, isym)
    g = bph.PotentialSolver(*grid)
    o = oracle_mod.Oracle(*grid)
    d_rho = torch.from_numpy(np.ascontiguousarray(rho.ravel(order="F"))).cuda()
    d_pot = torch.empty_like(d_rho)
    eps, seed = 0.01, 777
    mass0 = interior_mass(rho, dr, numphi)
    host = rho
    for it in range(4):
        tstep = 0 if it == 0 else it + 1
        mass = -1.0 if it == 0 else mass0
        g.scf_step(d_rho, d_pot, eps, mass, seed, it, tstep)
        g.synchronize()
        host, target = scf_update(host, eps, mass, seed, it, dr)
        m_dev, _ = g.scf_mass()
        assert m_dev == pytest.approx(target, rel=1e-13)
        dev_rho = d_rho.cpu().numpy().reshape(rho.shape, order="F")
        assert rel_l2(dev_rho, host) <= 1e-14, it
        assert interior_mass(dev_rho, dr, numphi) == pytest.approx(mass0, rel=1e-12)
        po = o.potential_solver(dev_rho, tstep)      # the oracle on the device's updated density
        assert rel_l2(d_pot.cpu().numpy().reshape(rho.shape, order="F"), po) <= 1e-12, it
        host = dev_rho                               # continue from the same density on both sides
    g.close()
    o.close()


def test_scf_step_rejects_bad_arguments(bph):
    import torch

    g = bph.PotentialSolver(18, 18, 16, 1.0 / 14.0, 2, 6)
    d = torch.zeros(18 * 18 * 16, dtype=torch.float64, device="cuda")
    with pytest.raises(bph.BphError):
        g.scf_step(d, d, -1.0, 0.0, 1, 0, 2)
    with pytest.raises(bph.BphError):
        g.scf_step(d, d, 0.01, float("nan"), 1, 0, 2)
    with pytest.raises(bph.BphError):
        g.scf_step(d, d, 0.01, 0.0, 1, -3, 2)
    g.close()
