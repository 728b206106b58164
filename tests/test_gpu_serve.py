"""Serving layer (bph_server_*): continuous batching of resident clients.

Every client's results must equal its own sequence of single potential_solver
calls (first cold, then warm), whether it is served alone or mixed with other
clients' requests, within the FP64 parity bound.
"""
import random
import time

import numpy as np
import pytest

from tests.helpers import rel_l2, smooth_density

pytestmark = pytest.mark.gpu

POT_TOL = 1e-12
GRID = (34, 26, 64, 1.0 / 30.0, 2, 30)


def _densities(nclients, nsteps, seed=0):
    numr, numz, numphi, dr, isym, _ = GRID
    out = []
    for c in range(nclients):
        base = smooth_density(numr, numz, numphi, dr, isym, seed=seed + c)
        out.append([np.asfortranarray(np.roll(base, t, axis=2) * (1.0 + 0.01 * t)) for t in range(nsteps)])
    return out


def _single_sequence(bph, seq):
    g = bph.PotentialSolver(*GRID)
    pots = [g.potential_solver(rho, 0 if t == 0 else t + 1) for t, rho in enumerate(seq)]
    g.close()
    return pots


def test_clients_match_their_single_sequences(bph):
    seqs = _densities(3, 3)
    g = bph.PotentialSolver(*GRID)
    srv = bph.Server(g, max_clients=4)
    clients = [srv.open_client() for _ in seqs]
    rids = {}
    for t in range(3):  # interleaved: every client's step t before step t+1
        for c, seq in zip(clients, seqs):
            rids[(c, t)] = srv.submit(c, seq[t])
    for c, seq in zip(clients, seqs):
        ref = _single_sequence(bph, seq)
        for t in range(3):
            pot, lat = srv.wait(rids[(c, t)], timeout=60.0)
            assert lat >= 0.0
            assert rel_l2(pot, ref[t]) <= POT_TOL, (c, t)
    st = srv.stats()
    assert st["solves"] == 9 and st["batches"] >= 3
    srv.close()
    g.close()


def test_result_same_alone_and_in_the_mix(bph):
    """Client A's potentials do not depend on which other requests share its batches."""
    seqs = _densities(5, 4, seed=10)
    # alone
    g = bph.PotentialSolver(*GRID)
    srv = bph.Server(g, max_clients=5)
    a = srv.open_client()
    alone = []
    for t in range(4):
        alone.append(srv.wait(srv.submit(a, seqs[0][t]), timeout=60.0)[0])
    srv.close()
    g.close()
    # mixed: the other four clients submit at random moments around A's requests
    g = bph.PotentialSolver(*GRID)
    srv = bph.Server(g, max_clients=5, max_batch=3)
    ids = [srv.open_client() for _ in range(5)]
    rng = random.Random(7)
    pending = []
    mine = []
    for t in range(4):
        for k in range(1, 5):
            if rng.random() < 0.7:
                pending.append(srv.submit(ids[k], seqs[k][t]))
        mine.append(srv.submit(ids[0], seqs[0][t]))
        time.sleep(rng.random() * 0.002)
    mixed = [srv.wait(r, timeout=60.0)[0] for r in mine]
    for r in pending:
        srv.wait(r, timeout=60.0)
    srv.close()
    g.close()
    for t in range(4):
        assert rel_l2(mixed[t], alone[t]) <= POT_TOL, t


def test_admission_by_memory_cap(bph):
    g = bph.PotentialSolver(*GRID)
    numr, numz, numphi = GRID[:3]
    ntot = numr * numz * numphi
    # about two clients' worth of device memory
    per = 8 * (ntot + (numr - 2) * (numz - 2) * numphi + 4 * ntot)
    srv = bph.Server(g, max_clients=16, mem_cap_bytes=2 * per)
    cap = srv.capacity
    assert 1 <= cap < 16
    got = [srv.open_client() for _ in range(cap)]
    assert len(set(got)) == cap
    with pytest.raises(bph.BphError) as ei:
        srv.open_client()
    assert ei.value.code == bph.BPH_ERR_NOMEM
    srv.close_client(got[0])
    assert srv.open_client() == got[0]  # the freed slot is admitted again
    srv.close()
    g.close()


def test_nonfinite_request_is_isolated(bph):
    seqs = _densities(2, 2, seed=20)
    g = bph.PotentialSolver(*GRID)
    srv = bph.Server(g, max_clients=2)
    a, b = srv.open_client(), srv.open_client()
    bad = seqs[0][0].copy(order="F")
    bad[5, 5, 5] = np.nan
    ra = srv.submit(a, bad)
    rb = srv.submit(b, seqs[1][0])
    with pytest.raises(bph.BphError) as ei:
        srv.wait(ra, timeout=60.0)
    assert ei.value.code == bph.BPH_ERR_NONFINITE
    ref_b = _single_sequence(bph, seqs[1])
    assert rel_l2(srv.wait(rb, timeout=60.0)[0], ref_b[0]) <= POT_TOL
    # the failed client starts again cold; the other continues warm
    ra2 = srv.submit(a, seqs[0][0])
    rb2 = srv.submit(b, seqs[1][1])
    ref_a = _single_sequence(bph, seqs[0])
    assert rel_l2(srv.wait(ra2, timeout=60.0)[0], ref_a[0]) <= POT_TOL
    assert rel_l2(srv.wait(rb2, timeout=60.0)[0], ref_b[1]) <= POT_TOL
    srv.close()
    g.close()


def test_poll_and_unknown_request(bph):
    seqs = _densities(1, 1, seed=30)
    g = bph.PotentialSolver(*GRID)
    srv = bph.Server(g, max_clients=1)
    c = srv.open_client()
    r = srv.submit(c, seqs[0][0])
    t0 = time.time()
    out = None
    while out is None and time.time() - t0 < 60.0:
        out = srv.poll(r)
    assert out is not None
    with pytest.raises(bph.BphError):
        srv.poll(r)  # reported done already
    srv.close()
    g.close()


def test_production_grid_batched_clients(bph):
    """130x98x256: 6 clients x 3 requests against each client's single sequence."""
    from bipoly_hydro_b200 import fields

    g = bph.PotentialSolver(130, 98, 256, 1.0 / 126.0, 2, 30)
    srv = bph.Server(g, max_clients=6)
    clients = [srv.open_client() for _ in range(6)]
    seqs = [[fields.rotate(fields.bipolytrope_pair(mass_ratio=0.3 + 0.1 * c), t) for t in range(3)]
            for c in range(6)]
    rids = {(c, t): srv.submit(c, seqs[c][t]) for t in range(3) for c in clients}
    res = {k: srv.wait(v, timeout=120.0)[0] for k, v in rids.items()}
    srv.close()
    g.close()
    ref_solver = bph.PotentialSolver(130, 98, 256, 1.0 / 126.0, 2, 30)
    for c in clients:
        for t in range(3):
            ref = ref_solver.potential_solver(seqs[c][t], 0 if t == 0 else t + 1)
            assert rel_l2(res[(c, t)], ref) <= POT_TOL, (c, t)
    ref_solver.close()


def test_device_array_mode_matches_host_mode(bph):
    import torch

    seqs = _densities(3, 3, seed=40)
    g = bph.PotentialSolver(*GRID)
    srv = bph.Server(g, max_clients=3, device_arrays=True)
    ids = [srv.open_client() for _ in seqs]
    d_rho = [[torch.from_numpy(np.ascontiguousarray(r.ravel(order="F"))).cuda() for r in seq] for seq in seqs]
    d_pot = [[torch.empty_like(x) for x in row] for row in d_rho]
    torch.cuda.synchronize()
    rids = {(c, t): srv.submit(c, d_rho[c][t], d_pot[c][t]) for t in range(3) for c in ids}
    for k, r in rids.items():
        srv.wait(r, timeout=60.0)
    srv.close()
    g.close()
    for c in ids:
        ref = _single_sequence(bph, seqs[c])
        for t in range(3):
            got = d_pot[c][t].cpu().numpy().reshape(ref[t].shape, order="F")
            assert rel_l2(got, ref[t]) <= POT_TOL, (c, t)


@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
def test_converged_mode_serves_converged_solutions(bph, mixed):
    """In converged mode (FP64 or FP32 refinement) every request's potential
    is the converged discrete solution of its density: equal to a single
    converged FP64 solve to 1e-9, first requests cold and later ones warm."""
    seqs = _densities(3, 3, seed=40)
    g = bph.PotentialSolver(*GRID)
    srv = bph.Server(g, max_clients=3)
    srv.set_converged(nsteps=10, tol=1e-12, max_cycles=80, mixed=mixed)
    clients = [srv.open_client() for _ in seqs]
    rids = {}
    for t in range(3):
        for c, seq in zip(clients, seqs):
            rids[(c, t)] = srv.submit(c, seq[t])
    ref = bph.PotentialSolver(*GRID)
    for c, seq in zip(clients, seqs):
        for t in range(3):
            pot, _ = srv.wait(rids[(c, t)], timeout=60.0)
            want, _ = ref.solve_converged(seq[t], 10, True, 1e-13, 200)
            assert rel_l2(pot, want) <= 1e-9, (c, t)
    srv.set_converged(0)  # back to the drop-in solve
    rid = srv.submit(clients[0], seqs[0][0])
    assert srv.wait(rid, timeout=60.0)[0].shape == seqs[0][0].shape
    srv.close()
    ref.close()
    g.close()
