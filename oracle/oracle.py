"""ctypes binding of the CPU oracle (oracle/bph_oracle.c).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
as the checker and by ``bench.py`` for its ``cpu_baseline`` leg and the
``--impl reference`` arm.  The product package never imports it.

Parity status: unpinned by the reference itself (it ships no golden vectors
and cannot be compiled here); pinned against analytic known answers in
tests/test_oracle_*.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc.so")
_lib = None


class OrcGrid(ctypes.Structure):
    _fields_ = [
        ("numr", ctypes.c_int),
        ("numz", ctypes.c_int),
        ("numphi", ctypes.c_int),
        ("dr", ctypes.c_double),
        ("isym", ctypes.c_int),
        ("mmax", ctypes.c_int),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        L.orc_setup.argtypes = [ctypes.POINTER(OrcGrid), ctypes.POINTER(vp)]
        L.orc_setup.restype = ctypes.c_int
        L.orc_destroy.argtypes = [vp]
        L.orc_potential_solver.argtypes = [vp, dp, dp, ctypes.c_int]
        L.orc_potential_solver.restype = ctypes.c_int
        L.orc_solve_nsteps.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_int]
        L.orc_solve_nsteps.restype = ctypes.c_int
        L.orc_solve_converged.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_int, ctypes.POINTER(ctypes.c_int), dp]
        L.orc_solve_converged.restype = ctypes.c_int
        L.orc_set_potential.argtypes = [vp, dp]
        L.orc_set_moments_override.argtypes = [vp, ctypes.c_void_p]
        L.orc_residual.argtypes = [vp, dp, dp]
        L.orc_residual.restype = ctypes.c_double
        L.orc_num_boundary_rows.argtypes = [vp]
        L.orc_num_boundary_rows.restype = ctypes.c_int
        L.orc_green.argtypes = [vp]
        L.orc_green.restype = dp
        L.orc_moments_S.argtypes = [vp]
        L.orc_moments_S.restype = dp
        L.orc_dt_schedule.argtypes = [vp, ctypes.c_int, dp]
        L.orc_slot_mode.argtypes = [vp, ctypes.c_int]
        L.orc_slot_mode.restype = ctypes.c_int
        for name in ("orc_gammln", "orc_ellf", "orc_elle"):
            getattr(L, name).argtypes = [ctypes.c_double]
            getattr(L, name).restype = ctypes.c_double
        for name in ("orc_rf", "orc_rd"):
            getattr(L, name).argtypes = [ctypes.c_double] * 3
            getattr(L, name).restype = ctypes.c_double
        L.orc_toroidal.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, dp]
        L.orc_realft.argtypes = [dp, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        L.orc_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def gammln(x: float) -> float:
    return lib().orc_gammln(float(x))


def rf(x, y, z) -> float:
    return lib().orc_rf(float(x), float(y), float(z))


def rd(x, y, z) -> float:
    return lib().orc_rd(float(x), float(y), float(z))


def ellf(k) -> float:
    return lib().orc_ellf(float(k))


def elle(k) -> float:
    return lib().orc_elle(float(k))


def toroidal(x: float, isym: int = 2, mmax: int = 30) -> np.ndarray:
    q = np.zeros(mmax)
    lib().orc_toroidal(float(x), int(isym), int(mmax), _dp(q))
    return q


def realft(col: np.ndarray, isign: int) -> np.ndarray:
    """realft on a copy of a 1-D float64 column."""
    d = np.ascontiguousarray(col, dtype=np.float64).copy()
    lib().orc_realft(_dp(d), 1, d.size, int(isign))
    return d


class Oracle:
    """One-rank CPU restatement of potsetup + potential_solver.

    Arrays are Fortran-ordered ``(numr, numz, numphi)`` float64, the layout of
    the reference's COMMON /poisson/ pot, rho (potential_solver.F90:18-19).
    """

    def __init__(self, numr: int, numz: int, numphi: int, dr: float, isym: int = 2, mmax: int = 30):
        self.shape = (numr, numz, numphi)
        self.grid = OrcGrid(numr, numz, numphi, float(dr), isym, mmax)
        self.isym, self.mmax, self.dr = isym, mmax, float(dr)
        h = ctypes.c_void_p()
        rc = lib().orc_setup(ctypes.byref(self.grid), ctypes.byref(h))
        if rc != 0:
            raise ValueError(f"orc_setup failed ({rc}): {lib().orc_last_error().decode()}")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, rho):
        rho = np.asfortranarray(rho, dtype=np.float64)
        if rho.shape != self.shape:
            raise ValueError(f"rho shape {rho.shape} != {self.shape}")
        return rho

    def _call(self, fn, rho, *args):
        rho = self._check(rho)
        pot = np.zeros(self.shape, dtype=np.float64, order="F")
        rc = fn(self._h, _dp(rho), _dp(pot), *args)
        if rc != 0:
            raise RuntimeError(f"oracle call failed ({rc}): {lib().orc_last_error().decode()}")
        return pot

    def potential_solver(self, rho, tstep: int):
        return self._call(lib().orc_potential_solver, rho, int(tstep))

    def solve_nsteps(self, rho, nsteps: int, cold: bool):
        return self._call(lib().orc_solve_nsteps, rho, int(nsteps), int(bool(cold)))

    def solve_converged(self, rho, nsteps: int = 20, cold: bool = True, tol: float = 1e-12,
                        max_cycles: int = 200):
        cyc = ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        pot = self._call(lib().orc_solve_converged, rho, int(nsteps), int(bool(cold)), float(tol),
                         int(max_cycles), ctypes.byref(cyc), ctypes.byref(res))
        return pot, cyc.value, res.value

    def set_potential(self, pot) -> None:
        p = np.asfortranarray(pot, dtype=np.float64)
        lib().orc_set_potential(self._h, _dp(p))

    def set_moments_override(self, S) -> None:
        """Test hook: later solves use these boundary moments S[m][b][2]
        (None: the contraction's own)."""
        if S is None:
            self._S_keep = None
            lib().orc_set_moments_override(self._h, None)
            return
        self._S_keep = np.ascontiguousarray(S, dtype=np.float64).copy()
        lib().orc_set_moments_override(self._h, self._S_keep.ctypes.data)

    def residual(self, rho, pot) -> float:
        rho = self._check(rho)
        pot = np.asfortranarray(pot, dtype=np.float64)
        return float(lib().orc_residual(self._h, _dp(rho), _dp(pot)))

    @property
    def nb(self) -> int:
        return int(lib().orc_num_boundary_rows(self._h))

    def green(self) -> np.ndarray:
        """Green tables G[m][b][p] (copy)."""
        nr, nz = self.shape[0] - 2, self.shape[1] - 2
        n = self.mmax * self.nb * nr * nz
        ptr = lib().orc_green(self._h)
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(self.mmax, self.nb, nr * nz).copy()

    def moments_S(self) -> np.ndarray:
        n = self.mmax * self.nb * 2
        ptr = lib().orc_moments_S(self._h)
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(self.mmax, self.nb, 2).copy()

    def dt_schedule(self, nsteps: int) -> np.ndarray:
        dt = np.zeros(nsteps)
        lib().orc_dt_schedule(self._h, int(nsteps), _dp(dt))
        return dt

    def slot_modes(self) -> np.ndarray:
        return np.array([lib().orc_slot_mode(self._h, i) for i in range(self.shape[2])])
