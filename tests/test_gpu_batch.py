"""Batched solves (bph_batch_*): n independent densities on one grid share one
pass over the Green tables; each instance keeps its own warm state.  Every
instance must equal its own single-solve sequence (and the oracle) to the
FP64 drop-in bar."""
import numpy as np
import pytest

from tests.helpers import rel_l2, smooth_density

pytestmark = pytest.mark.gpu


def _densities(grid, n):
    numr, numz, numphi, dr, isym, _ = grid
    return [np.asfortranarray(smooth_density(numr, numz, numphi, dr, isym, seed=100 + i) * (1.0 + 0.1 * i))
            for i in range(n)]


@pytest.mark.parametrize("grid", [(34, 26, 64, 1.0 / 30.0, 2, 30), (20, 14, 32, 1.0 / 18.0, 1, 8),
                                  (35, 21, 64, 1.0 / 31.0, 2, 12)], ids=["34x26x64", "isym1", "odd"])
def test_batch_equals_single_solves(oracle_mod, bph, grid):
    n = 5
    rhos = _densities(grid, n)
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=8)
    singles = [bph.PotentialSolver(*grid) for _ in range(n)]
    oracles = [oracle_mod.Oracle(*grid) for _ in range(2)]
    for tstep in (0, 2, 3):
        if tstep:
            rhos = [np.asfortranarray(np.roll(r, 1, axis=2)) for r in rhos]
        got = batch.solve(rhos, tstep)
        for i in range(n):
            want = singles[i].potential_solver(rhos[i], tstep)
            assert rel_l2(got[i], want) <= 1e-12, (tstep, i)
        for i in range(2):
            assert rel_l2(got[i], oracles[i].potential_solver(rhos[i], tstep)) <= 1e-12, (tstep, i)
    batch.close()
    for s in singles:
        s.close()
    solver.close()


def test_batch_subset_keeps_other_states(bph):
    """Solving instances 0..1 of a batch leaves instance 2's warm state alone."""
    grid = (34, 26, 64, 1.0 / 30.0, 2, 30)
    rhos = _densities(grid, 3)
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=3)
    ref = [bph.PotentialSolver(*grid) for _ in range(3)]
    batch.solve(rhos, 0)
    for i in range(3):
        ref[i].potential_solver(rhos[i], 0)
    batch.solve(rhos[:2], 2)
    for i in range(2):
        ref[i].potential_solver(rhos[i], 2)
    got = batch.solve(rhos, 3)
    for i in range(3):
        assert rel_l2(got[i], ref[i].potential_solver(rhos[i], 3)) <= 1e-12, i
    batch.close()
    solver.close()


def test_batch_production_grid_device_arrays(bph):
    import torch

    from bipoly_hydro_b200 import fields

    grid = (130, 98, 256, 1.0 / 126.0, 2, 30)
    n = 4
    rhos = [fields.bipolytrope_pair(mass_ratio=q) for q in (0.3, 0.5, 0.7, 1.0)]
    solver = bph.PotentialSolver(*grid)
    solver.set_stream(torch.cuda.current_stream())
    batch = bph.Batch(solver, capacity=n)
    d_rho = [torch.from_numpy(np.ascontiguousarray(r.ravel(order="F"))).cuda() for r in rhos]
    d_pot = [torch.empty_like(x) for x in d_rho]
    singles = [bph.PotentialSolver(*grid) for _ in range(n)]
    for tstep in (0, 2):
        batch.solve_device(d_rho, d_pot, tstep)
        solver.synchronize()
        for i in range(n):
            want = singles[i].potential_solver(rhos[i], tstep)
            got = d_pot[i].cpu().numpy().reshape(rhos[i].shape, order="F")
            assert rel_l2(got, want) <= 1e-12, (tstep, i)
    batch.close()
    solver.close()


def test_batch_rejects_bad_sizes(bph):
    grid = (18, 18, 16, 1.0 / 14.0, 2, 6)
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=2)
    rhos = _densities(grid, 3)
    with pytest.raises(bph.BphError):
        batch.solve(rhos, 0)
    batch.close()
    solver.close()


@pytest.mark.parametrize("grid", [(66, 66, 64, 1.0 / 62.0, 2, 30), (202, 152, 16, 1.0 / 200.0, 2, 4)],
                         ids=["66x66x64", "grid-wide-adi"])
def test_batch_converged_equals_single_converged(bph, grid):
    """Converged batched solves (FP64, and the FP32 refinement: on-chip kernels
    or, for slots beyond shared memory, the grid-wide ones) against single
    converged FP64 solves of each instance: cold, then warm after the
    densities move."""
    n = 3
    rhos = _densities(grid, n)
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=n)
    mixed_batch = bph.Batch(solver, capacity=n)  # its own warm states
    singles = [bph.PotentialSolver(*grid) for _ in range(n)]
    for cold in (True, False):
        if not cold:
            rhos = [np.asfortranarray(np.roll(r, 1, axis=2) * 1.01) for r in rhos]
        want = [singles[i].solve_converged(rhos[i], 10, cold, 1e-13, 80)[0] for i in range(n)]
        got, info = batch.solve_converged(rhos, nsteps=10, cold=cold, tol=1e-13, max_cycles=80)
        assert 1 <= info.cycles <= 80 and info.residual < 1e-8
        for i in range(n):
            assert rel_l2(got[i], want[i]) <= 1e-10, (cold, i)
        gm, _ = mixed_batch.solve_converged(rhos, nsteps=10, cold=cold, tol=1e-12, max_cycles=80, mixed=True)
        for i in range(n):
            assert rel_l2(gm[i], want[i]) <= 1e-9, ("mixed", cold, i)
    mixed_batch.close()
    for s in singles:
        s.close()
    batch.close()
    solver.close()


@pytest.mark.parametrize("n", [1, 4, 5, 16, 33], ids=lambda n: f"n{n}")
def test_tensor_core_contraction_matches_single_solve_moments(bph, n):
    """The batched boundary contraction (FP64 tensor cores, DMMA) gives every
    position the boundary moments S of its own single solve to 1e-13, at
    every batch size (33 positions: two column blocks of the kernel)."""
    grid = (34, 26, 64, 1.0 / 30.0, 2, 30)
    rhos = _densities(grid, n)
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=n)
    batch.solve(rhos, 0)
    got = batch.moments_S(n)
    single = bph.PotentialSolver(*grid)
    for i in range(n):
        single.potential_solver(rhos[i], 0)
        assert rel_l2(got[i], single.moments_S()) <= 1e-13, i
    single.close()
    batch.close()
    solver.close()


def test_tensor_core_contraction_production_grid(bph):
    """130x98x256, 16 positions: S per position against its single solve."""
    from bipoly_hydro_b200 import fields

    grid = (130, 98, 256, 1.0 / 126.0, 2, 30)
    n = 16
    rhos = [fields.bipolytrope_pair(mass_ratio=0.2 + 0.05 * i) for i in range(n)]
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=n)
    batch.solve(rhos, 0)
    got = batch.moments_S(n)
    single = bph.PotentialSolver(*grid)
    for i in range(0, n, 5):
        single.potential_solver(rhos[i], 0)
        assert rel_l2(got[i], single.moments_S()) <= 1e-13, i
    single.close()
    batch.close()
    solver.close()


@pytest.mark.parametrize("grid", [(202, 152, 16, 1.0 / 200.0, 2, 4), (35, 27, 32, 1.0 / 31.0, 2, 12),
                                  (100, 70, 32, 1.0 / 96.0, 1, 8)],
                         ids=["np30000-mmax4", "odd-np", "isym1"])
def test_tensor_core_contraction_slice_boundaries(bph, grid):
    """Grids whose zone slices are not whole multiples of the kernel's staged
    chunk (30000 zones in 12 slices, an odd zone count, the isym 1 bottom
    rows): S per position against its single solve to 1e-13."""
    n = 3
    rhos = _densities(grid, n)
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=n)
    batch.solve(rhos, 0)
    got = batch.moments_S(n)
    single = bph.PotentialSolver(*grid)
    for i in range(n):
        single.potential_solver(rhos[i], 0)
        assert rel_l2(got[i], single.moments_S()) <= 1e-13, i
    single.close()
    batch.close()
    solver.close()


def test_context_and_batch_destroyed_in_either_order(bph):
    """A garbage-collected host may release the context's handle before a
    batch on it: the batch keeps the device state alive, still solves, and
    frees it when it is destroyed."""
    grid = (34, 26, 64, 1.0 / 30.0, 2, 30)
    rhos = _densities(grid, 2)
    solver = bph.PotentialSolver(*grid)
    batch = bph.Batch(solver, capacity=2)
    ref = bph.Batch(solver, capacity=2)
    ref.solve(rhos, 0)
    want = ref.solve(rhos, 2)
    ref.close()
    batch.solve(rhos, 0)
    lib, h = solver._lib, solver._h
    solver._h = None
    solver._dependents = ()
    assert lib.bph_destroy(h) == 0
    got = batch.solve(rhos, 2)
    for i in range(2):
        assert rel_l2(got[i], want[i]) <= 1e-13, i
    batch.close()
