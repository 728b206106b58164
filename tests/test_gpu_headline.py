"""Oracle parity at the production grids the benchmark measures.

130x98x256 (dr = 1/126, isym 2, mmax 30) is the time-step workload: the
bipolytrope pair, a cold solve and then warm solves with the density rotated
by one azimuthal zone per call (potential_solver.F90:80-94 with
main.F90:396).  These tests run it through the same calls and the same
launch configuration as the benchmark (the warp-cooperative on-chip ADI,
the side stream for the slots without boundary data, programmatic
dependent launch, 8-column FFT tiles) and compare every potential with the oracle at the FP64
bar: relative L2 error <= 1e-12 with the same ADI step count.

258x194x64 has the production slot size of the 258x194 grids (256 x 192
interior zones per slot): its slots exceed shared memory, so the drop-in
takes the grid-wide panel ADI kernels.
"""
import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

POT_TOL = 1e-12
GRID_130 = (130, 98, 256, 1.0 / 126.0, 2, 30)


@pytest.fixture(scope="module")
def oracle_130(oracle_mod):
    o = oracle_mod.Oracle(*GRID_130)
    yield o
    o.close()


@pytest.fixture(scope="module")
def pair_rho():
    from bipoly_hydro_b200 import fields

    return fields.bipolytrope_pair()


def test_time_step_sequence_host_arrays(oracle_130, pair_rho, bph):
    """bph_potential_solver (host arrays): cold, then four warm rotated solves."""
    from bipoly_hydro_b200 import fields

    g = bph.PotentialSolver(*GRID_130)
    info = g.info()
    assert info["adi_kernel"] == bph.solver.ADI_KERNEL_WARP, info
    rho = pair_rho
    for tstep in range(0, 5):
        po = oracle_130.potential_solver(rho, tstep)
        pg = g.potential_solver(rho, tstep)
        err = rel_l2(pg, po)
        assert err <= POT_TOL, (tstep, err)
        if tstep == 0:
            assert rel_l2(g.moments_S(), oracle_130.moments_S()) <= 1e-13
        rho = fields.rotate(rho)
    g.close()


def test_time_step_sequence_device_arrays(oracle_130, pair_rho, bph):
    """bph_potential_solver_device on the caller's torch stream: the benchmark's
    call, with the free-slot ADI on the low-priority side stream and
    programmatic dependent launch; several solves are enqueued back to back
    before the host waits."""
    import torch

    from bipoly_hydro_b200 import fields

    torch.cuda.set_device(0)
    g = bph.PotentialSolver(*GRID_130)
    stream = torch.cuda.Stream()
    g.set_stream(stream)
    rhos = [fields.rotate(pair_rho, i) for i in range(5)]
    d_rho = [torch.from_numpy(np.ascontiguousarray(r.ravel(order="F"))).cuda() for r in rhos]
    d_pot = [torch.empty_like(d_rho[0]) for _ in rhos]
    torch.cuda.synchronize()
    for i in range(5):
        g.potential_solver_device(d_rho[i], d_pot[i], 0 if i == 0 else i + 1)
    g.synchronize()
    for i in range(5):
        po = oracle_130.potential_solver(rhos[i], 0 if i == 0 else i + 1)
        pg = d_pot[i].cpu().numpy().reshape(rhos[i].shape, order="F")
        err = rel_l2(pg, po)
        assert err <= POT_TOL, (i, err)
    g.close()


def test_warm_state_restored_from_previous_potential(oracle_130, pair_rho, bph):
    """The benchmark's parity check: the oracle's warm state set from the GPU's
    previous potential reproduces the GPU's next warm solve."""
    from bipoly_hydro_b200 import fields

    g = bph.PotentialSolver(*GRID_130)
    p0 = g.potential_solver(pair_rho, 0)
    rho1 = fields.rotate(pair_rho)
    p1 = g.potential_solver(rho1, 2)
    oracle_130.set_potential(p0)
    po = oracle_130.potential_solver(rho1, 2)
    assert rel_l2(p1, po) <= POT_TOL
    g.close()


def test_converged_fp64_and_mixed_match_oracle(oracle_130, pair_rho, bph):
    """bph_solve_converged against orc_solve_converged with the same cycle
    count, and the mixed-precision form within 1e-9 of the oracle."""
    g = bph.PotentialSolver(*GRID_130)
    po, co, ro = oracle_130.solve_converged(pair_rho, 10, True, 1e-11, 60)
    pg, info = g.solve_converged(pair_rho, 10, True, 1e-11, 60)
    assert info.cycles == co, (info.cycles, co)
    assert rel_l2(pg, po) <= POT_TOL
    assert abs(info.residual - ro) <= 0.5 * ro + 1e-12
    pm, im = g.solve_converged_mixed(pair_rho, 10, True, 1e-11, 60)
    assert rel_l2(pm, po) <= 1e-9, (rel_l2(pm, po), im.cycles)
    g.close()


def test_grid_wide_adi_at_production_slot_size(oracle_mod, bph):
    """258x194x64, dr = 1/250, mmax 30: slots of 256 x 192 zones take the
    grid-wide panel ADI; cold and warm solves at the FP64 bar."""
    from bipoly_hydro_b200 import fields

    grid = (258, 194, 64, 1.0 / 250.0, 2, 30)
    g = bph.PotentialSolver(*grid)
    assert g.info()["adi_threads"] == 0
    o = oracle_mod.Oracle(*grid)
    rho = fields.bipolytrope_pair(258, 194, 64, 1.0 / 250.0)
    for tstep in (0, 2, 3):
        err = rel_l2(g.potential_solver(rho, tstep), o.potential_solver(rho, tstep))
        assert err <= POT_TOL, (tstep, err)
        rho = fields.rotate(rho)
    o.close()
    g.close()


@pytest.mark.parametrize("kernel", ["warp", "segmented"])
def test_both_on_chip_adi_kernels_match_oracle(oracle_130, pair_rho, bph, monkeypatch, kernel):
    """The warp-cooperative ADI (default on this grid) and the CTA-wide
    segmented one (BPH_ADI_WARP=0 at set-up) both meet the bar, cold and warm,
    including the converged form whose cycles report update norms."""
    from bipoly_hydro_b200 import fields

    monkeypatch.setenv("BPH_ADI_WARP", "1" if kernel == "warp" else "0")
    g = bph.PotentialSolver(*GRID_130)
    want = bph.solver.ADI_KERNEL_WARP if kernel == "warp" else bph.solver.ADI_KERNEL_SEGMENTED
    assert g.info()["adi_kernel"] == want
    rho = pair_rho
    for tstep in (0, 2):
        err = rel_l2(g.potential_solver(rho, tstep), oracle_130.potential_solver(rho, tstep))
        assert err <= POT_TOL, (kernel, tstep, err)
        rho = fields.rotate(rho)
    po, co, _ = oracle_130.solve_converged(pair_rho, 10, True, 1e-11, 60)
    pg, info = g.solve_converged(pair_rho, 10, True, 1e-11, 60)
    assert info.cycles == co and rel_l2(pg, po) <= POT_TOL
    g.close()


def test_warp_refinement_kernel_matches_oracle(oracle_130, pair_rho, bph):
    """The FP32 warp-cooperative refinement kernel (mixed kind 4): cold and
    warm converged mixed solves within 1e-9 of the oracle's converged FP64
    potential, single and batched."""
    from bipoly_hydro_b200 import fields

    g = bph.PotentialSolver(*GRID_130)
    g.set_mixed_adi(bph.solver.MIXED_ADI_WARP)
    po, _, _ = oracle_130.solve_converged(pair_rho, 10, True, 1e-12, 60)
    pm, im = g.solve_converged_mixed(pair_rho, 10, True, 1e-12, 60)
    assert rel_l2(pm, po) <= 1e-9, (rel_l2(pm, po), im.cycles)
    rho2 = fields.rotate(pair_rho)
    po2, _, _ = oracle_130.solve_converged(rho2, 10, False, 1e-12, 60)
    pm2, im2 = g.solve_converged_mixed(rho2, 10, False, 1e-12, 60)
    assert rel_l2(pm2, po2) <= 1e-9, (rel_l2(pm2, po2), im2.cycles)
    batch = bph.Batch(g, capacity=3)
    rhos = [fields.rotate(pair_rho, i) for i in range(3)]
    pots, info = batch.solve_converged(rhos, 10, True, 1e-12, 60, mixed=True)
    ref = oracle_130.solve_converged(rhos[2], 10, True, 1e-12, 60)[0]
    assert rel_l2(pots[2], ref) <= 1e-9, rel_l2(pots[2], ref)
    batch.close()
    g.close()


def test_sm_partitioned_solve_matches_oracle(oracle_130, pair_rho, bph, monkeypatch):
    """BPH_GREEN=1: the overlapped solve with the contraction and the
    free-slot ADI on disjoint SM partitions (green contexts) gives the same
    potentials: cold and warm solves at the FP64 bar, device arrays."""
    import torch

    from bipoly_hydro_b200 import fields

    monkeypatch.setenv("BPH_GREEN", "1")
    monkeypatch.setenv("BPH_GREEN_SMS", "64")
    g = bph.PotentialSolver(*GRID_130)
    if g.info()["green_sms"] <= 0:
        step = -g.info()["green_sms"]
        g.close()
        pytest.skip(f"the driver offers no SM partitions on this device (set-up step {step})")
    assert g.info()["green_sms"] >= 64
    rhos = [fields.rotate(pair_rho, i) for i in range(3)]
    d_rho = [torch.from_numpy(np.ascontiguousarray(r.ravel(order="F"))).cuda() for r in rhos]
    d_pot = [torch.empty_like(d_rho[0]) for _ in rhos]
    for i in range(3):
        g.potential_solver_device(d_rho[i], d_pot[i], 0 if i == 0 else i + 1)
    g.synchronize()
    for i in range(3):
        po = oracle_130.potential_solver(rhos[i], 0 if i == 0 else i + 1)
        assert rel_l2(d_pot[i].cpu().numpy().reshape(rhos[i].shape, order="F"), po) <= POT_TOL, i
    g.close()


def test_setup_autotune_keeps_the_faster_candidates(bph, monkeypatch):
    """bph_setup times both boundary contractions, both FFT tile variants and
    both FP64 ADI kernels on the grid and keeps the faster of each (reported
    by bph_info); BPH_AUTOTUNE=0 keeps the defaults and times nothing."""
    S = bph.solver
    g = bph.PotentialSolver(*GRID_130)
    i = g.info()
    g.close()
    assert i["contract_full_ns"] > 0 and i["contract_compact_ns"] > 0, i
    want = S.CONTRACT_COMPACT if i["contract_compact_ns"] <= i["contract_full_ns"] else S.CONTRACT_FULL
    assert i["contract_kind"] == want, i
    assert i["fft_ns"] > 0 and i["fft_dense_ns"] > 0, i
    assert i["fft_dense"] == (1 if i["fft_dense_ns"] < i["fft_ns"] else 0), i
    assert i["adi_seg_ns"] > 0 and i["adi_warp_ns"] > 0, i
    want = S.ADI_KERNEL_SEGMENTED if i["adi_seg_ns"] < i["adi_warp_ns"] else S.ADI_KERNEL_WARP
    assert i["adi_kernel"] == want, i
    monkeypatch.setenv("BPH_AUTOTUNE", "0")
    g = bph.PotentialSolver(*GRID_130)
    i = g.info()
    g.close()
    assert i["contract_full_ns"] == 0 and i["fft_ns"] == 0 and i["adi_seg_ns"] == 0, i
    assert i["contract_kind"] == S.CONTRACT_COMPACT and i["adi_kernel"] == S.ADI_KERNEL_WARP and i["fft_dense"] == 0


def test_direct_refinement_at_the_production_grid(oracle_130, pair_rho, bph):
    """MIXED_DIRECT at 130x98x256: cold and warm converged solves and a
    converged batch within 1e-9 of the oracle's converged FP64 potentials."""
    from bipoly_hydro_b200 import fields

    g = bph.PotentialSolver(*GRID_130)
    g.set_mixed_adi(bph.solver.MIXED_DIRECT)
    po, co, _ = oracle_130.solve_converged(pair_rho, 10, True, 1e-12, 60)
    pm, im = g.solve_converged_mixed(pair_rho, 10, True, 1e-12, 60)
    assert rel_l2(pm, po) <= 1e-9, (rel_l2(pm, po), im.cycles, co)
    rho2 = fields.rotate(pair_rho)
    po2, _, _ = oracle_130.solve_converged(rho2, 10, False, 1e-12, 60)
    pm2, im2 = g.solve_converged_mixed(rho2, 10, False, 1e-12, 60)
    assert rel_l2(pm2, po2) <= 1e-9, (rel_l2(pm2, po2), im2.cycles)
    batch = bph.Batch(g, capacity=3)
    rhos = [fields.rotate(pair_rho, i) for i in range(3)]
    pots, info = batch.solve_converged(rhos, 10, True, 1e-12, 60, mixed=True)
    for i in (0, 2):
        ref = oracle_130.solve_converged(rhos[i], 10, True, 1e-12, 60)[0]
        assert rel_l2(pots[i], ref) <= 1e-9, (i, rel_l2(pots[i], ref), info.cycles)
    batch.close()
    g.close()
