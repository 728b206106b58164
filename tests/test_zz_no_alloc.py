"""bph_green_contract_noalloc: the boundary contraction for callers that
cannot allocate device memory (its scratch is a file-scope device array).

Its boundary moments S must equal those the regular solve computes for the
same density (bph_copy_moments after a solve) and the CPU oracle's, on two
calls in a row (the second call reuses the scratch the first one left
behind); a 3x3 interior (9 zones, fewer than the 16 splits) exercises the
clamp of the split count to the zone count.  This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import rel_l2, smooth_density

pytestmark = pytest.mark.gpu

S_TOL = 1e-12


def _moments(torch, rho, numphi, mmax, fm):
    """Interior moments mom[m][cos|sin][p] = sum_l rho (cos|sin)(fm m (l - 1/2) dphi), FP64."""
    numr, numz, _ = rho.shape
    interior = np.ascontiguousarray(rho[1:-1, 1:-1, :].reshape(-1, numphi, order="F"))  # (np, N)
    l = np.arange(numphi, dtype=np.float64) + 0.5
    ang = np.outer(l, fm * np.arange(mmax, dtype=np.float64)) * (2.0 * np.pi / numphi)  # (N, mmax)
    r = torch.from_numpy(interior).cuda()
    c = r @ torch.from_numpy(np.cos(ang)).cuda()  # (np, mmax)
    s = r @ torch.from_numpy(np.sin(ang)).cuda()
    mom = torch.stack([c.T, s.T], dim=1).contiguous()  # (mmax, 2, np)
    return mom


@pytest.mark.parametrize("grid", [(34, 26, 64, 1.0 / 30.0, 2, 30), (130, 98, 256, 1.0 / 126.0, 2, 30),
                                  (20, 14, 32, 1.0 / 18.0, 1, 8), (18, 16, 32, 1.0 / 16.0, 3, 6),
                                  (5, 5, 16, 1.0 / 3.0, 2, 2), (21, 13, 16, 1.0 / 19.0, 2, 4)],
                         ids=["34x26x64", "130x98x256", "isym1", "isym3", "np9-split-clamp", "odd-np"])
def test_noalloc_contraction_matches_solve(bph, oracle_mod, grid):
    import torch

    numr, numz, numphi, dr, isym, mmax = grid
    solver = bph.PotentialSolver(*grid)
    rho = smooth_density(numr, numz, numphi, dr, isym)
    solver.potential_solver(rho, 0)          # the existing entry point
    s_ref = solver.moments_S()
    o = oracle_mod.Oracle(*grid)             # the same moments from the CPU oracle
    o.potential_solver(rho, 0)
    s_orc = o.moments_S()
    o.close()
    mom = _moments(torch, rho, numphi, mmax, 2 if isym == 3 else 1)
    lib = bph.load_library()
    torch.cuda.synchronize()
    for call in range(2):
        d_s = torch.full((mmax * solver.nb * 2,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.bph_green_contract_noalloc(solver._h, ctypes.c_void_p(mom.data_ptr()),
                                            ctypes.c_void_p(d_s.data_ptr()))
        assert rc == 0, lib.bph_last_error().decode()
        solver.synchronize()
        s_new = d_s.cpu().numpy().reshape(mmax, solver.nb, 2)
        assert np.all(np.isfinite(s_new)), f"call {call}"
        assert rel_l2(s_new, s_ref) <= S_TOL, f"call {call}: {rel_l2(s_new, s_ref):.3e}"
        assert rel_l2(s_new, s_orc) <= S_TOL, f"call {call} vs oracle: {rel_l2(s_new, s_orc):.3e}"
    solver.close()


def test_noalloc_rejects_null_arguments(bph):
    lib = bph.load_library()
    assert lib.bph_green_contract_noalloc(None, None, None) == bph.BPH_ERR_INVALID
