"""What a reduced-precision boundary contraction would do to the potential.

The mixed-precision form keeps the boundary contraction S = G^T M (the
tables against the density moments, bessel.F90:186-296) in FP64.  This
test records why, on the CPU with the oracle: the contraction is computed
in numpy the way a tensor-core kernel would compute it --
  * BF16x3: two-term BF16 splits of both operands, the three leading
    products exact in FP32, FP32 accumulation;
  * TF32x3: the same with TF32 (10 explicit mantissa bits);
  * an Ozaki split: per-row / per-column power-of-two scaling, k INT8
    slices per operand, exact integer slice products (INT8 tensor cores
    with INT32 accumulation), FP64 recombination --
and the oracle then solves with that S in place of its own
(orc_set_moments_override).  Measured on 66x66x64 (two n=1 polytropes,
converged solves), relative L2 change of S / of the potential:
  FP64 in numpy        2.8e-15 / 3.8e-14
  BF16x3               2.9e-7  / 5.5e-8
  TF32x3               1.6e-7  / 1.8e-8
  Ozaki INT8, 5 slices 3.4e-10 / 2.0e-10
  Ozaki INT8, 6 slices 2.1e-12 / 1.2e-12
  Ozaki INT8, 7 slices 2.8e-15 / 4.0e-14
The BF16 and TF32 splits miss the 1e-9 bar of the mixed form (the
boundary data are Dirichlet values that no refinement of the interior
corrects); an Ozaki split meets it from 5 slices and matches FP64 at 7.
"""
import numpy as np
import pytest

from tests.helpers import rel_l2

GRID = (66, 66, 64, 1.0 / 62.0, 2, 30)


def _round_bits(x, keep):
    """Round float32 values to `keep` explicit mantissa bits (nearest even)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    drop = 23 - keep
    half = (1 << (drop - 1)) - 1
    u = (u + half + ((u >> drop) & 1)) & ~np.uint64((1 << drop) - 1) & np.uint64(0xFFFFFFFF)
    return u.astype(np.uint32).view(np.float32)


def _split2(x, keep):
    hi = _round_bits(x, keep)
    lo = _round_bits(x - hi.astype(np.float64), keep)
    return hi, lo


def contract_split3(G, M, keep):
    """S = G @ M with two-term splits of `keep` mantissa bits and FP32 accumulation."""
    gh, gl = _split2(G, keep)
    mh, ml = _split2(M, keep)
    s = (gh @ mh).astype(np.float32) + (gh @ ml).astype(np.float32) + (gl @ mh).astype(np.float32)
    return s.astype(np.float64)


def _slices(x, axis, k):
    """INT8 slices of x scaled per row (axis=1) or per column (axis=0)."""
    amax = np.max(np.abs(x), axis=axis, keepdims=True)
    amax[amax == 0] = 1.0
    e = np.ceil(np.log2(amax))
    r = x / np.exp2(e)
    out = []
    for _ in range(k):
        r = r * 128.0
        q = np.clip(np.rint(r), -127, 127)
        out.append(q.astype(np.int64))
        r = r - q
    return out, e


def contract_ozaki(G, M, k):
    qg, eg = _slices(G, 1, k)
    qm, em = _slices(M, 0, k)
    s = np.zeros((G.shape[0], M.shape[1]))
    for t in range(k):
        for u in range(k - t):
            s += (qg[t] @ qm[u]).astype(np.float64) * 2.0 ** (-7 * (t + u + 2))
    return s * np.exp2(eg) * np.exp2(em)


def moments(rho, mmax):
    numr, numz, numphi = rho.shape
    interior = rho[1:-1, 1:-1, :].reshape(-1, numphi, order="F")  # (np, N)
    ang = np.outer(np.arange(numphi) + 0.5, np.arange(mmax)) * (2.0 * np.pi / numphi)
    return interior @ np.cos(ang), interior @ np.sin(ang)  # (np, mmax) each


@pytest.fixture(scope="module")
def setup(oracle_mod):
    from bipoly_hydro_b200 import fields

    o = oracle_mod.Oracle(*GRID)
    rho = fields.two_polytropes()
    pot_ref, _, _ = o.solve_converged(rho, 20, True, 1e-13, 200)
    G = o.green()  # [m][b][p]
    mc, ms = moments(rho, GRID[5])
    yield o, rho, pot_ref, G, mc, ms
    o.close()


def _solve_with(o, rho, G, mc, ms, contract):
    mmax, nb = G.shape[0], G.shape[1]
    S = np.zeros((mmax, nb, 2))
    for m in range(mmax):
        M = np.stack([mc[:, m], ms[:, m]], axis=1)
        S[m] = contract(G[m], M)
    S[0, :, 1] = 0.0
    o.set_moments_override(S)
    pot, _, _ = o.solve_converged(rho, 20, True, 1e-13, 200)
    o.set_moments_override(None)
    return S, pot


def test_fp64_contraction_reproduces_the_oracle(setup):
    o, rho, pot_ref, G, mc, ms = setup
    S, pot = _solve_with(o, rho, G, mc, ms, lambda g, m: g @ m)
    assert rel_l2(pot, pot_ref) <= 1e-13


@pytest.mark.parametrize("name,keep,floor", [("bf16x3", 7, 1e-9), ("tf32x3", 10, 1e-9)])
def test_split_contractions_miss_the_mixed_bar(setup, name, keep, floor):
    o, rho, pot_ref, G, mc, ms = setup
    S, pot = _solve_with(o, rho, G, mc, ms, lambda g, m: contract_split3(g, m, keep))
    err = rel_l2(pot, pot_ref)
    assert err > floor, (name, err)


@pytest.mark.parametrize("k,bar", [(5, 1e-9), (7, 1e-12)])
def test_ozaki_int8_split_meets_the_bar(setup, k, bar):
    o, rho, pot_ref, G, mc, ms = setup
    S, pot = _solve_with(o, rho, G, mc, ms, lambda g, m: contract_ozaki(g, m, k))
    err = rel_l2(pot, pot_ref)
    assert err <= bar, (k, err)
