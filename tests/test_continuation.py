"""The reference's continuation record (ritecont_frac_new.F90:151-160):
one Fortran unformatted sequential record holding s, t, a, rho, tau, pot,
tempa, frac1, frac2 as real(8) (numr, numz, numphi) arrays, framed by
4-byte length markers.  bph_read_continuation reads rho and pot back
(host code: these tests need no GPU); the GPU test restores the warm state
from such a file and checks the next warm solve against the oracle."""
import numpy as np
import pytest

from tests.helpers import rel_l2, smooth_density

SHAPE = (14, 12, 16)


def _arrays(seed=3):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(rng.standard_normal(SHAPE)) for _ in range(9)]


def write_record(path, arrays, byteorder="<", subrecord=None):
    """What gfortran writes for `write(12) s, t, a, rho, tau, pot, tempa, frac1, frac2`
    (subrecord: split the payload into subrecords of at most that many bytes,
    the convention for records beyond 2 GiB)."""
    payload = b"".join(np.asarray(a, dtype=byteorder + "f8").tobytes(order="F") for a in arrays)
    chunks = [payload] if subrecord is None else [payload[i:i + subrecord] for i in range(0, len(payload), subrecord)]
    with open(path, "wb") as f:
        for k, ch in enumerate(chunks):
            lead = len(ch) if k == len(chunks) - 1 else -len(ch)
            f.write(np.array([lead], dtype=byteorder + "i4").tobytes())
            f.write(ch)
            f.write(np.array([len(ch)], dtype=byteorder + "i4").tobytes())


@pytest.mark.parametrize("byteorder,subrecord", [("<", None), (">", None), ("<", 1000)],
                         ids=["little-endian", "big-endian", "subrecords"])
def test_reads_rho_and_pot_of_the_record(bph, tmp_path, byteorder, subrecord):
    arrays = _arrays()
    path = str(tmp_path / "fort.12.100.0")
    write_record(path, arrays, byteorder, subrecord)
    rho, pot = bph.read_continuation(path, *SHAPE)
    assert np.array_equal(rho, arrays[3])
    assert np.array_equal(pot, arrays[5])


def test_rejects_a_record_of_another_grid(bph, tmp_path):
    path = str(tmp_path / "fort.12.1.0")
    write_record(path, _arrays())
    with pytest.raises(bph.BphError) as ei:
        bph.read_continuation(path, 14, 12, 32)
    assert ei.value.code == bph.BPH_ERR_INVALID


def test_rejects_truncated_and_missing_files(bph, tmp_path):
    path = tmp_path / "fort.12.2.0"
    write_record(str(path), _arrays())
    data = path.read_bytes()
    path.write_bytes(data[:-100])
    with pytest.raises(bph.BphError):
        bph.read_continuation(str(path), *SHAPE)
    with pytest.raises(bph.BphError):
        bph.read_continuation(str(tmp_path / "absent"), *SHAPE)


@pytest.mark.gpu
def test_restart_from_record_continues_warm(bph, oracle_mod, tmp_path):
    """A run writes its state; a new context restores it and its next warm
    solve equals the oracle's warm solve from the same potential."""
    grid = (34, 26, 64, 1.0 / 30.0, 2, 30)
    numr, numz, numphi, dr, isym, _ = grid
    rho = smooth_density(numr, numz, numphi, dr, isym)
    o = oracle_mod.Oracle(*grid)
    pot = o.solve_nsteps(rho, 20, True)
    zeros = np.zeros_like(rho)
    path = str(tmp_path / "fort.12.500.0")
    write_record(path, [zeros, zeros, zeros, rho, zeros, pot, zeros, zeros, zeros])
    g = bph.PotentialSolver(*grid)
    rho_back = g.restore_continuation(path)
    assert np.array_equal(rho_back, rho)
    rho2 = np.asfortranarray(np.roll(rho, 1, axis=2))
    o.set_potential(pot)
    assert rel_l2(g.potential_solver(rho2, 501), o.potential_solver(rho2, 501)) <= 1e-12
    g.close()
    o.close()
