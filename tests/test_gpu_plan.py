"""Batches on grids too large for the on-chip ADI kernel, and plans: batches
on several grids recorded as one CUDA graph whose branches run concurrently.
Every instance must equal its own single-solve sequence to the FP64 drop-in
bar, whichever way it was launched."""
import numpy as np
import pytest

from tests.helpers import rel_l2, smooth_density

pytestmark = pytest.mark.gpu

LARGE = (202, 152, 16, 1.0 / 200.0, 2, 4)  # 200 x 150 interior: slots beyond shared memory


def _densities(grid, n, seed=300):
    numr, numz, numphi, dr, isym, _ = grid
    return [np.asfortranarray(smooth_density(numr, numz, numphi, dr, isym, seed=seed + i) * (1.0 + 0.2 * i))
            for i in range(n)]


def test_large_grid_batch_equals_single_solves(bph):
    n = 3
    rhos = _densities(LARGE, n)
    solver = bph.PotentialSolver(*LARGE)
    assert solver.info()["adi_threads"] == 0
    batch = bph.Batch(solver, capacity=4)
    singles = [bph.PotentialSolver(*LARGE) for _ in range(n)]
    for tstep in (0, 2, 3):
        if tstep:
            rhos = [np.asfortranarray(np.roll(r, 1, axis=2)) for r in rhos]
        got = batch.solve(rhos, tstep)
        for i in range(n):
            assert rel_l2(got[i], singles[i].potential_solver(rhos[i], tstep)) <= 1e-12, (tstep, i)
    # a subset in another order: the instance map of the grid-wide kernels
    rhos = [np.asfortranarray(np.roll(r, 1, axis=2)) for r in rhos]
    got = batch.solve_instances([2, 0], [rhos[2], rhos[0]], 4)
    assert rel_l2(got[0], singles[2].potential_solver(rhos[2], 4)) <= 1e-12
    assert rel_l2(got[1], singles[0].potential_solver(rhos[0], 4)) <= 1e-12
    for s in singles:
        s.close()
    batch.close()
    solver.close()


def _plan_setup(bph, torch, grids, counts):
    parts, singles, host = [], [], []
    for g, n in zip(grids, counts):
        solver = bph.PotentialSolver(*g)
        solver.set_stream(torch.cuda.current_stream())
        batch = bph.Batch(solver, capacity=n)
        rhos = _densities(g, n, seed=400 + 10 * len(parts))
        d_rho = [torch.from_numpy(np.ascontiguousarray(r.ravel(order="F"))).cuda() for r in rhos]
        d_pot = [torch.empty_like(x) for x in d_rho]
        parts.append((batch, d_rho, d_pot))
        singles.append([bph.PotentialSolver(*g) for _ in range(n)])
        host.append(rhos)
    return parts, singles, host


def test_plan_of_mixed_grids_equals_single_solves(bph):
    import torch

    grids = [(34, 26, 64, 1.0 / 30.0, 2, 30), (66, 66, 64, 1.0 / 62.0, 2, 30), LARGE]
    counts = [3, 2, 2]
    parts, singles, host = _plan_setup(bph, torch, grids, counts)
    plan = bph.Plan(parts)
    stream = torch.cuda.Stream()
    for tstep in (0, 2, 3):
        if tstep:
            host = [[np.asfortranarray(np.roll(r, 1, axis=2)) for r in rs] for rs in host]
        for (batch, d_rho, _), rs in zip(parts, host):
            for d, r in zip(d_rho, rs):
                d.copy_(torch.from_numpy(np.ascontiguousarray(r.ravel(order="F"))))
        stream.wait_stream(torch.cuda.current_stream())
        plan.launch(tstep, stream)
        plan.synchronize(stream)
        for p, ((batch, _, d_pot), rs) in enumerate(zip(parts, host)):
            for i, r in enumerate(rs):
                got = d_pot[i].cpu().numpy().reshape(r.shape, order="F")
                want = singles[p][i].potential_solver(r, tstep)
                assert rel_l2(got, want) <= 1e-12, (tstep, p, i)
    assert plan.launches > 0
    plan.close()
    for (batch, _, _), ss in zip(parts, singles):
        for s in ss:
            s.close()
        batch.solver.close()


def test_plan_reports_non_finite_density(bph):
    import torch

    grids = [(34, 26, 64, 1.0 / 30.0, 2, 30), (35, 21, 64, 1.0 / 31.0, 2, 12)]
    parts, singles, _ = _plan_setup(bph, torch, grids, [2, 1])
    plan = bph.Plan(parts)
    parts[1][1][0][9 + 35 * (9 + 21 * 2)] = float("nan")  # interior zone (J, K, L) = (10, 10, 3)
    torch.cuda.synchronize()
    plan.launch(0)
    with pytest.raises(bph.BphError) as err:
        plan.synchronize()
    assert err.value.code == bph.BPH_ERR_NONFINITE
    plan.close()
    for (batch, _, _), ss in zip(parts, singles):
        for s in ss:
            s.close()
        batch.solver.close()


def test_plan_rejects_shared_context(bph):
    import torch

    g = (34, 26, 64, 1.0 / 30.0, 2, 30)
    solver = bph.PotentialSolver(*g)
    batch = bph.Batch(solver, capacity=2)
    d = [torch.zeros(34 * 26 * 64, dtype=torch.float64, device="cuda") for _ in range(2)]
    with pytest.raises(bph.BphError):
        bph.Plan([(batch, d[:1], d[1:]), (batch, d[:1], d[1:])])
    with pytest.raises(bph.BphError):
        bph.Plan([(batch, d * 2, d * 2)])  # 4 positions > capacity 2
    batch.close()
    solver.close()


def test_contexts_set_up_largest_first_keep_working(bph):
    """Kernel shared-memory limits are process-wide: a context set up later
    for a smaller grid must not break the larger one set up before it."""
    big = (66, 66, 64, 1.0 / 62.0, 2, 30)
    rho = _densities(big, 1)[0]
    a = bph.PotentialSolver(*big)
    want = a.potential_solver(rho, 0)
    smaller = [bph.PotentialSolver(*g) for g in [(34, 26, 64, 1.0 / 30.0, 2, 30), (35, 21, 64, 1.0 / 31.0, 2, 12),
                                                 (18, 18, 16, 1.0 / 14.0, 2, 6)]]
    b = bph.Batch(a, capacity=2)
    got = b.solve([rho, rho], 0)
    assert rel_l2(a.potential_solver(rho, 0), want) == 0.0
    assert rel_l2(got[0], want) <= 1e-12 and rel_l2(got[1], want) <= 1e-12
    b.close()
    for s in smaller:
        s.close()
    a.close()


def test_large_grid_server_mixed_converged(bph):
    """Serving on a grid whose slots exceed shared memory, in mixed converged
    mode: the grid-wide FP32 refinement runs on client slots through the
    instance map; every result is the converged FP64 solution to 1e-9."""
    rhos = _densities(LARGE, 3, seed=500)
    g = bph.PotentialSolver(*LARGE)
    srv = bph.Server(g, max_clients=3)
    srv.set_converged(nsteps=10, tol=1e-12, max_cycles=80, mixed=True)
    clients = [srv.open_client() for _ in range(3)]
    rids = [srv.submit(clients[2], rhos[2]), srv.submit(clients[0], rhos[0])]
    rhos2 = [np.asfortranarray(np.roll(r, 1, axis=2)) for r in rhos]
    rids.append(srv.submit(clients[0], rhos2[0]))  # warm, after the first request of client 0
    ref = bph.PotentialSolver(*LARGE)
    for rid, rho in zip(rids, [rhos[2], rhos[0], rhos2[0]]):
        pot, _ = srv.wait(rid, timeout=120.0)
        want, _ = ref.solve_converged(rho, 10, True, 1e-13, 200)
        assert rel_l2(pot, want) <= 1e-9
    srv.close()
    ref.close()
    g.close()
