"""Host-side mirror of the reference's solver interface over the C ABI.

The reference exposes two argument-less Fortran subroutines that share COMMON
blocks: ``potsetup`` (potsetup.F90:6) builds the Green tables and ADI
coefficients once, and ``potential_solver`` (potential_solver.F90:6) turns
``rho`` into ``pot`` every time step.  :class:`PotentialSolver` keeps the same
two operations with the COMMON state made explicit: constructing it is
``potsetup``, :meth:`PotentialSolver.potential_solver` is the per-step call
with the same ``tstep`` warm/cold rule.

All computation runs in ``libbph.so`` (CUDA, sm_100a).  There is no CPU path:
if the library or a CUDA device is missing, construction raises.
"""
from __future__ import annotations

import ctypes
import weakref
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbph.so")

BPH_OK = 0
BPH_ERR_INVALID = -1
BPH_ERR_NOMEM = -2
BPH_ERR_NONFINITE = -3
BPH_ERR_CUDA = -4
BPH_ERR_TIMEOUT = -5
BPH_ERR_STATE = -6

_ERR_NAMES = {
    BPH_ERR_INVALID: "BPH_ERR_INVALID",
    BPH_ERR_NOMEM: "BPH_ERR_NOMEM",
    BPH_ERR_NONFINITE: "BPH_ERR_NONFINITE",
    BPH_ERR_CUDA: "BPH_ERR_CUDA",
    BPH_ERR_TIMEOUT: "BPH_ERR_TIMEOUT",
    BPH_ERR_STATE: "BPH_ERR_STATE",
}

#: Every symbol include/bph.h declares, in declaration order.
EXPORTED_SYMBOLS = (
    "bph_setup", "bph_potential_solver", "bph_potential_solver_device", "bph_solve_nsteps",
    "bph_solve_converged", "bph_potential_solver_phieff", "bph_set_potential", "bph_solve_converged_mixed", "bph_set_stream", "bph_synchronize", "bph_destroy", "bph_last_error",
    "bph_version", "bph_num_boundary_rows", "bph_copy_green", "bph_copy_moments", "bph_run_phase",
    "bph_green_contract_noalloc", "bph_info", "bph_configure", "bph_launch_count", "bph_device_bytes",
    "bph_batch_create", "bph_batch_solve", "bph_batch_solve_instances", "bph_batch_solve_converged",
    "bph_batch_destroy",
    "bph_batch_device_bytes", "bph_plan_create", "bph_plan_launch", "bph_plan_synchronize", "bph_plan_launches",
    "bph_plan_destroy",
    "bph_server_create", "bph_server_set_converged", "bph_server_capacity", "bph_server_open_client",
    "bph_server_close_client",
    "bph_server_submit", "bph_server_poll", "bph_server_wait", "bph_server_stats", "bph_server_destroy",
    "bph_register_host", "bph_unregister_host", "bph_read_continuation", "bph_restore_continuation",
    "bph_scf_step", "bph_scf_mass", "bph_batch_copy_moments",
)

#: bph_configure keys and values.
CFG_MIXED_ADI = 0
MIXED_ADI_AUTO, MIXED_ADI_FORWARD, MIXED_ADI_INCREMENT, MIXED_ADI_GLOBAL, MIXED_ADI_WARP = 0, 1, 2, 3, 4
MIXED_DIRECT = 5  # the defect equation solved directly in FP32 (not an ADI)

#: bph_info(BPH_INFO_ADI_KERNEL) values.
ADI_KERNEL_WARP, ADI_KERNEL_SEGMENTED, ADI_KERNEL_ONCHIP, ADI_KERNEL_GRID_WIDE = 1, 2, 3, 4
CONTRACT_FULL, CONTRACT_COMPACT = 1, 2
# bph_info keys in index order: BPH_INFO_<KEY> of include/bph.h, lower case
INFO_KEYS = ("adi_threads", "adi_smem", "mixed_threads", "mixed_smem", "mixed_ctas_per_sm", "contract_split",
             "mixed_kind", "mixed_forward_ns", "mixed_increment_ns", "adi_prefetch", "adi_kernel", "adi_warp_smem",
             "mixed_warp_ns", "green_sms", "contract_kind", "fft_dense", "contract_full_ns", "contract_compact_ns",
             "fft_ns", "fft_dense_ns", "adi_seg_ns", "adi_warp_ns", "mixed_direct_ns")

#: bph_run_phase phase ids.
PHASE_FFT_RHO, PHASE_CONTRACT, PHASE_SLOTS, PHASE_ADI, PHASE_FFT_INV = range(5)


class BphError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {message}")
        self.code = code


class Grid(ctypes.Structure):
    """``bph_grid_t``: the runhydro.h / pot.h / fort.7 parameters of the solve."""

    _fields_ = [
        ("numr", ctypes.c_int),
        ("numz", ctypes.c_int),
        ("numphi", ctypes.c_int),
        ("dr", ctypes.c_double),
        ("isym", ctypes.c_int),
        ("mmax", ctypes.c_int),
    ]


_lib = None


def load_library(path: str | None = None):
    """Load libbph.so and declare its prototypes.  Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is not built; run `make -C bipoly_hydro_b200/csrc` (the solver has no CPU fallback)")
    L = ctypes.CDLL(p)
    vp, dp, i, sz = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    L.bph_setup.argtypes = [ctypes.POINTER(Grid), ctypes.POINTER(vp)]
    L.bph_potential_solver.argtypes = [vp, dp, dp, i]
    L.bph_potential_solver_device.argtypes = [vp, dp, dp, i]
    L.bph_solve_nsteps.argtypes = [vp, dp, dp, i, i, i]
    L.bph_solve_converged.argtypes = [vp, dp, dp, i, i, ctypes.c_double, i, i, ctypes.POINTER(i),
                                      ctypes.POINTER(ctypes.c_double)]
    L.bph_potential_solver_phieff.argtypes = [vp, dp, dp, dp, ctypes.c_double, i, i]
    L.bph_potential_solver_phieff.restype = ctypes.c_int
    L.bph_set_potential.argtypes = [vp, dp, i]
    L.bph_set_potential.restype = ctypes.c_int
    L.bph_solve_converged_mixed.argtypes = L.bph_solve_converged.argtypes
    L.bph_solve_converged_mixed.restype = ctypes.c_int
    L.bph_set_stream.argtypes = [vp, vp]
    L.bph_synchronize.argtypes = [vp]
    L.bph_destroy.argtypes = [vp]
    L.bph_last_error.restype = ctypes.c_char_p
    L.bph_version.restype = ctypes.c_char_p
    L.bph_num_boundary_rows.argtypes = [vp]
    L.bph_copy_green.argtypes = [vp, dp, sz]
    L.bph_copy_moments.argtypes = [vp, dp, sz]
    L.bph_run_phase.argtypes = [vp, i, dp, dp, i]
    L.bph_green_contract_noalloc.argtypes = [vp, dp, dp]
    L.bph_green_contract_noalloc.restype = ctypes.c_int
    L.bph_batch_create.argtypes = [vp, i, ctypes.POINTER(vp)]
    L.bph_batch_create.restype = ctypes.c_int
    L.bph_batch_solve.argtypes = [vp, i, ctypes.POINTER(vp), ctypes.POINTER(vp), i, i]
    L.bph_batch_solve.restype = ctypes.c_int
    L.bph_batch_solve_instances.argtypes = [vp, i, ctypes.POINTER(i), ctypes.POINTER(vp), ctypes.POINTER(vp), i, i]
    L.bph_batch_solve_instances.restype = ctypes.c_int
    L.bph_batch_solve_converged.argtypes = [vp, i, ctypes.POINTER(vp), ctypes.POINTER(vp), i, i, ctypes.c_double, i,
                                            i, i, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_double)]
    L.bph_batch_solve_converged.restype = ctypes.c_int
    L.bph_batch_copy_moments.argtypes = [vp, i, dp, sz]
    L.bph_batch_copy_moments.restype = ctypes.c_int
    L.bph_batch_destroy.argtypes = [vp]
    L.bph_batch_destroy.restype = ctypes.c_int
    ll, dbl = ctypes.c_longlong, ctypes.c_double
    L.bph_server_create.argtypes = [vp, i, sz, i, i, ctypes.POINTER(vp)]
    L.bph_server_set_converged.argtypes = [vp, i, dbl, i, i]
    L.bph_server_capacity.argtypes = [vp]
    L.bph_server_open_client.argtypes = [vp, ctypes.POINTER(i)]
    L.bph_server_close_client.argtypes = [vp, i]
    L.bph_server_submit.argtypes = [vp, i, dp, dp, ctypes.POINTER(ll)]
    L.bph_server_poll.argtypes = [vp, ll, ctypes.POINTER(dbl)]
    L.bph_server_wait.argtypes = [vp, ll, dbl, ctypes.POINTER(dbl)]
    L.bph_server_stats.argtypes = [vp, ctypes.POINTER(ll), ctypes.POINTER(ll)]
    L.bph_server_destroy.argtypes = [vp]
    for name in ("bph_server_create", "bph_server_set_converged", "bph_server_capacity", "bph_server_open_client",
                 "bph_server_close_client", "bph_server_submit", "bph_server_poll", "bph_server_wait", "bph_server_stats",
                 "bph_server_destroy"):
        getattr(L, name).restype = ctypes.c_int
    L.bph_plan_create.argtypes = [i, ctypes.POINTER(vp), ctypes.POINTER(i), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                  ctypes.POINTER(vp)]
    L.bph_plan_launch.argtypes = [vp, i, vp]
    L.bph_plan_synchronize.argtypes = [vp, vp]
    L.bph_plan_launches.argtypes = [vp]
    L.bph_plan_destroy.argtypes = [vp]
    for name in ("bph_plan_create", "bph_plan_launch", "bph_plan_synchronize", "bph_plan_launches",
                 "bph_plan_destroy"):
        getattr(L, name).restype = ctypes.c_int
    L.bph_batch_device_bytes.argtypes = [vp]
    L.bph_batch_device_bytes.restype = ctypes.c_size_t
    L.bph_info.argtypes = [vp, i]
    L.bph_info.restype = ctypes.c_longlong
    L.bph_configure.argtypes = [vp, i, i]
    L.bph_configure.restype = i
    L.bph_launch_count.argtypes = [vp]
    L.bph_launch_count.restype = ctypes.c_longlong
    L.bph_device_bytes.argtypes = [vp]
    L.bph_device_bytes.restype = ctypes.c_size_t
    L.bph_scf_step.argtypes = [vp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong, i, i]
    L.bph_scf_step.restype = i
    L.bph_scf_mass.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.bph_scf_mass.restype = i
    L.bph_read_continuation.argtypes = [ctypes.c_char_p, ctypes.POINTER(Grid), dp, dp]
    L.bph_read_continuation.restype = i
    L.bph_restore_continuation.argtypes = [vp, ctypes.c_char_p, dp]
    L.bph_restore_continuation.restype = i
    L.bph_register_host.argtypes = [vp, sz]
    L.bph_register_host.restype = i
    L.bph_unregister_host.argtypes = [vp]
    L.bph_unregister_host.restype = i
    for name in ("bph_setup", "bph_potential_solver", "bph_potential_solver_device", "bph_solve_nsteps",
                 "bph_solve_converged", "bph_set_stream", "bph_synchronize", "bph_destroy",
                 "bph_num_boundary_rows", "bph_copy_green", "bph_copy_moments", "bph_run_phase"):
        getattr(L, name).restype = ctypes.c_int
    if path is None:
        _lib = L
    return L


def _check(rc: int) -> None:
    if rc != BPH_OK:
        raise BphError(rc, load_library().bph_last_error().decode(errors="replace"))


def _host_ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _dev_ptr(x) -> int:
    """Device address of a torch CUDA tensor, an object with data_ptr(), or an int."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    raise TypeError("expected a device pointer (int) or a CUDA tensor")


@dataclass
class ConvergedInfo:
    cycles: int
    residual: float


class PotentialSolver:
    """potsetup + potential_solver for one grid on the current CUDA device.

    ``rho``/``pot`` are ``(numr, numz, numphi)`` float64 arrays in Fortran
    order, guard zones included (the reference's COMMON /poisson/ layout).
    """

    def __init__(self, numr: int, numz: int, numphi: int, dr: float, isym: int = 2, mmax: int = 30):
        self._lib = load_library()
        self._dependents = weakref.WeakSet()
        self.grid = Grid(int(numr), int(numz), int(numphi), float(dr), int(isym), int(mmax))
        self.shape = (int(numr), int(numz), int(numphi))
        self.isym, self.mmax, self.dr = int(isym), int(mmax), float(dr)
        h = ctypes.c_void_p()
        _check(self._lib.bph_setup(ctypes.byref(self.grid), ctypes.byref(h)))
        self._h = h

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        # batches and servers on this context go first (they hold its device state)
        for dep in list(getattr(self, "_dependents", ())):
            dep.close()
        if getattr(self, "_h", None):
            self._lib.bph_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return int(self._h.value)

    # -- host-array API -----------------------------------------------------
    def _rho_host(self, rho) -> np.ndarray:
        a = np.asarray(rho, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"rho has shape {a.shape}, expected {self.shape}")
        return np.asfortranarray(a)

    def potential_solver(self, rho, tstep: int, out: np.ndarray | None = None) -> np.ndarray:
        """potential_solver.F90:6-109: tstep > 1 warm (5 ADI steps), else cold (20)."""
        r = self._rho_host(rho)
        pot = out if out is not None else np.empty(self.shape, dtype=np.float64, order="F")
        if not pot.flags.f_contiguous or pot.dtype != np.float64 or pot.shape != self.shape:
            raise ValueError("out must be a Fortran-ordered float64 array of the grid shape")
        _check(self._lib.bph_potential_solver(self._h, _host_ptr(r), _host_ptr(pot), int(tstep)))
        return pot

    def potential_solver_phieff(self, rho, tstep: int, omega_frame: float):
        """potential_solver plus phieff = pot - 0.5 omega^2 rhf^2 (source.F90:156)."""
        r = self._rho_host(rho)
        pot = np.empty(self.shape, dtype=np.float64, order="F")
        phieff = np.empty(self.shape, dtype=np.float64, order="F")
        _check(self._lib.bph_potential_solver_phieff(self._h, _host_ptr(r), _host_ptr(pot), _host_ptr(phieff),
                                                     float(omega_frame), int(tstep), 0))
        return pot, phieff

    def set_potential(self, pot) -> None:
        """Warm state from a (checkpointed) potential for the next tstep > 1 solve."""
        a = np.asfortranarray(np.asarray(pot, dtype=np.float64))
        if a.shape != self.shape:
            raise ValueError(f"pot has shape {a.shape}, expected {self.shape}")
        _check(self._lib.bph_set_potential(self._h, _host_ptr(a), 0))

    def restore_continuation(self, path: str) -> np.ndarray:
        """Warm state from the reference's continuation record (fort.12.<tstep>.<rank>,
        ritecont_frac_new.F90:151-160); returns the density stored beside it."""
        rho = np.empty(self.shape, dtype=np.float64, order="F")
        _check(self._lib.bph_restore_continuation(self._h, os.fsencode(path), _host_ptr(rho)))
        return rho

    def solve_nsteps(self, rho, nsteps: int, cold: bool) -> np.ndarray:
        r = self._rho_host(rho)
        pot = np.empty(self.shape, dtype=np.float64, order="F")
        _check(self._lib.bph_solve_nsteps(self._h, _host_ptr(r), _host_ptr(pot), int(nsteps), int(bool(cold)), 0))
        return pot

    def solve_converged(self, rho, nsteps: int = 20, cold: bool = True, tol: float = 1e-13,
                        max_cycles: int = 200):
        r = self._rho_host(rho)
        pot = np.empty(self.shape, dtype=np.float64, order="F")
        cyc, res = ctypes.c_int(0), ctypes.c_double(0.0)
        _check(self._lib.bph_solve_converged(self._h, _host_ptr(r), _host_ptr(pot), int(nsteps), int(bool(cold)),
                                             float(tol), int(max_cycles), 0, ctypes.byref(cyc), ctypes.byref(res)))
        return pot, ConvergedInfo(cyc.value, res.value)

    def solve_converged_mixed(self, rho, nsteps: int = 20, cold: bool = True, tol: float = 1e-13,
                              max_cycles: int = 200):
        """FP32 ADI cycles with FP64 residual/update refinement to the converged solution."""
        r = self._rho_host(rho)
        pot = np.empty(self.shape, dtype=np.float64, order="F")
        cyc, res = ctypes.c_int(0), ctypes.c_double(0.0)
        _check(self._lib.bph_solve_converged_mixed(self._h, _host_ptr(r), _host_ptr(pot), int(nsteps),
                                                   int(bool(cold)), float(tol), int(max_cycles), 0,
                                                   ctypes.byref(cyc), ctypes.byref(res)))
        return pot, ConvergedInfo(cyc.value, res.value)

    def solve_converged_device(self, d_rho, d_pot, nsteps: int = 20, cold: bool = True, tol: float = 1e-13,
                               max_cycles: int = 200, mixed: bool = False) -> ConvergedInfo:
        """Converged solve on device arrays (synchronous: convergence is checked on the host)."""
        fn = self._lib.bph_solve_converged_mixed if mixed else self._lib.bph_solve_converged
        cyc = ctypes.c_int(0)
        _check(fn(self._h, _dev_ptr(d_rho), _dev_ptr(d_pot), int(nsteps), int(bool(cold)), float(tol),
                  int(max_cycles), 1, ctypes.byref(cyc), None))
        return ConvergedInfo(cyc.value, float("nan"))

    # -- device-array API ---------------------------------------------------
    def set_stream(self, stream) -> None:
        """Run later work on a CUDA stream: an int handle or a torch.cuda.Stream
        (0 / None is CUDA's default stream)."""
        handle = 0
        if stream is not None:
            handle = stream if isinstance(stream, int) else int(stream.cuda_stream)
        _check(self._lib.bph_set_stream(self._h, ctypes.c_void_p(handle or None)))

    def potential_solver_device(self, d_rho, d_pot, tstep: int) -> None:
        """Enqueue one solve on device arrays (pointers or CUDA tensors)."""
        _check(self._lib.bph_potential_solver_device(self._h, _dev_ptr(d_rho), _dev_ptr(d_pot), int(tstep)))

    def scf_step(self, d_rho, d_pot, eps: float = 0.01, mass: float = 0.0, seed: int = 20261203,
                 iteration: int = 0, tstep: int = 2) -> None:
        """One SCF-like iteration on device arrays (bph_scf_step): the seeded
        density update rho <- 0.9 rho + 0.1 rho (1 + eps xi), renormalised to
        `mass` (<= 0: its mass before the update), then potential_solver."""
        _check(self._lib.bph_scf_step(self._h, _dev_ptr(d_rho), _dev_ptr(d_pot), float(eps), float(mass),
                                      int(seed) & 0xFFFFFFFFFFFFFFFF, int(iteration), int(tstep)))

    def scf_mass(self):
        """(target mass, renormalisation factor) of the last scf_step."""
        m, sc = ctypes.c_double(0.0), ctypes.c_double(0.0)
        _check(self._lib.bph_scf_mass(self._h, ctypes.byref(m), ctypes.byref(sc)))
        return m.value, sc.value

    def solve_nsteps_device(self, d_rho, d_pot, nsteps: int, cold: bool) -> None:
        _check(self._lib.bph_solve_nsteps(self._h, _dev_ptr(d_rho), _dev_ptr(d_pot), int(nsteps),
                                          int(bool(cold)), 1))

    def synchronize(self) -> None:
        _check(self._lib.bph_synchronize(self._h))

    # -- inspection ---------------------------------------------------------
    @property
    def nb(self) -> int:
        return int(self._lib.bph_num_boundary_rows(self._h))

    def green(self) -> np.ndarray:
        nr, nz = self.shape[0] - 2, self.shape[1] - 2
        out = np.empty(self.mmax * self.nb * nr * nz, dtype=np.float64)
        _check(self._lib.bph_copy_green(self._h, _host_ptr(out), out.size))
        return out.reshape(self.mmax, self.nb, nr * nz)

    def moments_S(self) -> np.ndarray:
        out = np.empty(self.mmax * self.nb * 2, dtype=np.float64)
        _check(self._lib.bph_copy_moments(self._h, _host_ptr(out), out.size))
        return out.reshape(self.mmax, self.nb, 2)

    def run_phase(self, phase: int, d_rho=None, d_pot=None, nsteps: int = 5) -> None:
        """Enqueue one kernel of the solve (timing diagnostics)."""
        _check(self._lib.bph_run_phase(self._h, int(phase), _dev_ptr(d_rho) if d_rho is not None else None,
                                       _dev_ptr(d_pot) if d_pot is not None else None, int(nsteps)))

    def info(self) -> dict:
        """Launch-configuration facts (bph_info)."""
        return {n: int(self._lib.bph_info(self._h, i)) for i, n in enumerate(INFO_KEYS)}

    def set_mixed_adi(self, kind: int) -> None:
        """Inner solver of the mixed form's refinement cycles: MIXED_ADI_AUTO
        (time every kind that fits and keep the fastest cycle), an FP32 ADI
        kernel (MIXED_ADI_FORWARD, MIXED_ADI_INCREMENT, MIXED_ADI_GLOBAL,
        MIXED_ADI_WARP) or MIXED_DIRECT (the defect equation solved directly)."""
        _check(self._lib.bph_configure(self._h, CFG_MIXED_ADI, int(kind)))

    @property
    def launch_count(self) -> int:
        return int(self._lib.bph_launch_count(self._h))

    @property
    def device_bytes(self) -> int:
        return int(self._lib.bph_device_bytes(self._h))


def read_continuation(path: str, numr: int, numz: int, numphi: int):
    """(rho, pot) of the reference's continuation record (bph_read_continuation),
    Fortran-ordered (numr, numz, numphi) arrays."""
    g = Grid(int(numr), int(numz), int(numphi), 1.0, 2, 2)
    rho = np.empty((numr, numz, numphi), dtype=np.float64, order="F")
    pot = np.empty_like(rho)
    _check(load_library().bph_read_continuation(os.fsencode(path), ctypes.byref(g), _host_ptr(rho), _host_ptr(pot)))
    return rho, pot


def register_host(a: np.ndarray) -> None:
    """Pin a host array for fast host-array solves (bph_register_host).  Call
    :func:`unregister_host` on the same array before it is freed."""
    if not isinstance(a, np.ndarray) or a.nbytes == 0:
        raise ValueError("expected a non-empty numpy array")
    _check(load_library().bph_register_host(ctypes.c_void_p(a.ctypes.data), a.nbytes))


def unregister_host(a: np.ndarray) -> None:
    _check(load_library().bph_unregister_host(ctypes.c_void_p(a.ctypes.data)))


def version() -> str:
    return load_library().bph_version().decode()


class Batch:
    """Up to ``capacity`` independent solves on one solver's grid (bph_batch_*).

    Instance i keeps its own warm state; one call solves instances 0..n-1 at
    the same ``tstep`` with a single pass over the shared Green tables.
    """

    def __init__(self, solver: PotentialSolver, capacity: int):
        self.solver = solver
        self._lib = solver._lib
        self.capacity = int(capacity)
        self._dependents = weakref.WeakSet()  # plans recording this batch
        solver._dependents.add(self)
        h = ctypes.c_void_p()
        _check(self._lib.bph_batch_create(solver._h, self.capacity, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        for dep in list(getattr(self, "_dependents", ())):
            dep.close()
        if getattr(self, "_h", None):
            self._lib.bph_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, rhos, tstep: int):
        """Host arrays: list of (numr, numz, numphi) densities -> list of potentials."""
        rs = [self.solver._rho_host(r) for r in rhos]
        pots = [np.empty(self.solver.shape, dtype=np.float64, order="F") for _ in rs]
        n = len(rs)
        arr_r = (ctypes.c_void_p * n)(*[a.ctypes.data for a in rs])
        arr_p = (ctypes.c_void_p * n)(*[a.ctypes.data for a in pots])
        _check(self._lib.bph_batch_solve(self._h, n, arr_r, arr_p, int(tstep), 0))
        return pots

    def solve_device(self, d_rhos, d_pots, tstep: int) -> None:
        """Device arrays (pointers or CUDA tensors), enqueued on the solver's stream."""
        n = len(d_rhos)
        arr_r = (ctypes.c_void_p * n)(*[_dev_ptr(x) for x in d_rhos])
        arr_p = (ctypes.c_void_p * n)(*[_dev_ptr(x) for x in d_pots])
        _check(self._lib.bph_batch_solve(self._h, n, arr_r, arr_p, int(tstep), 1))

    def solve_instances(self, instances, rhos, tstep: int):
        """Host arrays for the distinct ``instances``; the others keep their state."""
        rs = [self.solver._rho_host(r) for r in rhos]
        pots = [np.empty(self.solver.shape, dtype=np.float64, order="F") for _ in rs]
        n = len(rs)
        idx = (ctypes.c_int * n)(*[int(v) for v in instances])
        arr_r = (ctypes.c_void_p * n)(*[a.ctypes.data for a in rs])
        arr_p = (ctypes.c_void_p * n)(*[a.ctypes.data for a in pots])
        _check(self._lib.bph_batch_solve_instances(self._h, n, idx, arr_r, arr_p, int(tstep), 0))
        return pots

    def _converged(self, arr_r, arr_p, n, nsteps, cold, tol, max_cycles, mixed, on_device):
        cyc, res = ctypes.c_int(0), ctypes.c_double(0.0)
        _check(self._lib.bph_batch_solve_converged(self._h, n, arr_r, arr_p, int(nsteps), int(bool(cold)), float(tol),
                                                   int(max_cycles), int(bool(mixed)), int(on_device),
                                                   ctypes.byref(cyc), ctypes.byref(res)))
        return ConvergedInfo(cyc.value, res.value)

    def solve_converged(self, rhos, nsteps: int = 10, cold: bool = False, tol: float = 1e-11, max_cycles: int = 100,
                        mixed: bool = False):
        """Host arrays: converged solves of instances 0..n-1 -> (potentials, ConvergedInfo)."""
        rs = [self.solver._rho_host(r) for r in rhos]
        pots = [np.empty(self.solver.shape, dtype=np.float64, order="F") for _ in rs]
        n = len(rs)
        arr_r = (ctypes.c_void_p * n)(*[a.ctypes.data for a in rs])
        arr_p = (ctypes.c_void_p * n)(*[a.ctypes.data for a in pots])
        info = self._converged(arr_r, arr_p, n, nsteps, cold, tol, max_cycles, mixed, 0)
        return pots, info

    def solve_converged_device(self, d_rhos, d_pots, nsteps: int = 10, cold: bool = False, tol: float = 1e-11,
                               max_cycles: int = 100, mixed: bool = False):
        """Device arrays: as solve_converged, results enqueued on the solver's stream."""
        n = len(d_rhos)
        arr_r = (ctypes.c_void_p * n)(*[_dev_ptr(x) for x in d_rhos])
        arr_p = (ctypes.c_void_p * n)(*[_dev_ptr(x) for x in d_pots])
        return self._converged(arr_r, arr_p, n, nsteps, cold, tol, max_cycles, mixed, 1)

    @property
    def device_bytes(self) -> int:
        return int(self._lib.bph_batch_device_bytes(self._h))

    def moments_S(self, n: int) -> np.ndarray:
        """Boundary moments S[pos][m][b][cos|sin] of positions 0..n-1 of the last call."""
        mmax, nb = self.solver.mmax, self.solver.nb
        out = np.empty(n * mmax * nb * 2, dtype=np.float64)
        _check(self._lib.bph_batch_copy_moments(self._h, int(n), _host_ptr(out), out.size))
        return out.reshape(n, mmax, nb, 2)


class Plan:
    """Batches on several grids recorded as one CUDA graph (bph_plan_*).

    ``parts`` is a list of ``(batch, d_rhos, d_pots)``: each batch on its own
    solver (grid), with device arrays (CUDA tensors or pointers) that stay
    fixed; refill the densities between launches.  ``launch`` replays every
    part's solves concurrently on ``stream`` (None: the default stream).
    """

    def __init__(self, parts):
        self._lib = parts[0][0]._lib
        self._keep = [(b, list(r), list(p)) for b, r, p in parts]  # arrays stay alive with the plan
        n = len(parts)
        batches = (ctypes.c_void_p * n)(*[b._h.value for b, _, _ in parts])
        counts = (ctypes.c_int * n)(*[len(r) for _, r, _ in parts])
        self._rows = [((ctypes.c_void_p * len(r))(*[_dev_ptr(x) for x in r]),
                       (ctypes.c_void_p * len(pp))(*[_dev_ptr(x) for x in pp])) for _, r, pp in parts]
        if any(len(r) != len(pp) for _, r, pp in parts):
            raise ValueError("every part needs as many potentials as densities")
        rho = (ctypes.c_void_p * n)(*[ctypes.cast(a, ctypes.c_void_p).value for a, _ in self._rows])
        pot = (ctypes.c_void_p * n)(*[ctypes.cast(b, ctypes.c_void_p).value for _, b in self._rows])
        h = ctypes.c_void_p()
        _check(self._lib.bph_plan_create(n, batches, counts, rho, pot, ctypes.byref(h)))
        self._h = h
        for b, _, _ in parts:
            b._dependents.add(self)

    @staticmethod
    def _stream(stream):
        if stream is None:
            return None
        return ctypes.c_void_p(getattr(stream, "cuda_stream", stream))

    def launch(self, tstep: int, stream=None) -> None:
        _check(self._lib.bph_plan_launch(self._h, int(tstep), self._stream(stream)))

    def synchronize(self, stream=None) -> None:
        _check(self._lib.bph_plan_synchronize(self._h, self._stream(stream)))

    @property
    def launches(self) -> int:
        """Kernel launches in one replay."""
        return int(self._lib.bph_plan_launches(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.bph_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


BPH_PENDING = 1


class Server:
    """Continuous batching of solve requests for resident clients (bph_server_*).

    Each client keeps its density transform and last potential on the device;
    its first request is cold, later ones warm-start from its previous
    potential.  ``submit`` returns at once; ``poll``/``wait`` report completion.
    The server drives the solver's context from a worker thread: make no other
    call on that solver while the server is open.
    """

    def __init__(self, solver: PotentialSolver, max_clients: int, mem_cap_bytes: int = 0, max_batch: int = 0,
                 device_arrays: bool = False):
        self.solver = solver
        self._lib = solver._lib
        self.device_arrays = bool(device_arrays)
        h = ctypes.c_void_p()
        _check(self._lib.bph_server_create(solver._h, int(max_clients), int(mem_cap_bytes), int(max_batch),
                                           1 if self.device_arrays else 0, ctypes.byref(h)))
        self._h = h
        self._live = {}  # request id -> (rho, pot) kept alive until completion
        solver._dependents.add(self)

    def set_converged(self, nsteps: int = 10, tol: float = 1e-11, max_cycles: int = 100, mixed: bool = False) -> None:
        """Serve converged solves (FP64, or mixed precision) from the next batch on; nsteps=0: drop-in."""
        _check(self._lib.bph_server_set_converged(self._h, int(nsteps), float(tol), int(max_cycles), int(bool(mixed))))

    @property
    def capacity(self) -> int:
        return int(self._lib.bph_server_capacity(self._h))

    def open_client(self) -> int:
        cid = ctypes.c_int(-1)
        _check(self._lib.bph_server_open_client(self._h, ctypes.byref(cid)))
        return cid.value

    def close_client(self, client: int) -> None:
        _check(self._lib.bph_server_close_client(self._h, int(client)))

    def submit(self, client: int, rho, pot=None) -> int:
        """Queue a solve; ``pot`` is written when the request completes.  Host
        mode: Fortran-ordered float64 arrays (pot allocated if None).  Device
        mode: CUDA tensors or device pointers, rho's writes complete.  Returns
        the request id."""
        if self.device_arrays:
            if pot is None:
                raise ValueError("device mode needs a pot array")
            r, p_ptr, r_ptr = rho, _dev_ptr(pot), _dev_ptr(rho)
        else:
            r = self.solver._rho_host(rho)
            if pot is None:
                pot = np.empty(self.solver.shape, dtype=np.float64, order="F")
            if not (pot.flags.f_contiguous and pot.dtype == np.float64 and pot.shape == self.solver.shape):
                raise ValueError("pot must be a Fortran-ordered float64 array of the grid's shape")
            r_ptr, p_ptr = _host_ptr(r), _host_ptr(pot)
        rid = ctypes.c_longlong(0)
        _check(self._lib.bph_server_submit(self._h, int(client), r_ptr, p_ptr, ctypes.byref(rid)))
        self._live[rid.value] = (r, pot)
        return rid.value

    def poll(self, request: int):
        """None while pending, else (pot, latency_s); raises BphError if it failed."""
        lat = ctypes.c_double(0.0)
        rc = self._lib.bph_server_poll(self._h, int(request), ctypes.byref(lat))
        if rc == BPH_PENDING:
            return None
        _, pot = self._live.pop(int(request), (None, None))
        _check(rc)
        return pot, lat.value

    def wait(self, request: int, timeout: float = 0.0):
        """(pot, latency_s) once the request completes; raises BphError if it failed or timed out."""
        lat = ctypes.c_double(0.0)
        rc = self._lib.bph_server_wait(self._h, int(request), float(timeout), ctypes.byref(lat))
        if rc == -5:  # BPH_ERR_TIMEOUT: still pending, keep its arrays alive
            _check(rc)
        _, pot = self._live.pop(int(request), (None, None))
        _check(rc)
        return pot, lat.value

    def stats(self):
        b, n = ctypes.c_longlong(0), ctypes.c_longlong(0)
        _check(self._lib.bph_server_stats(self._h, ctypes.byref(b), ctypes.byref(n)))
        return {"batches": b.value, "solves": n.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.bph_server_destroy(self._h)
            self._h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
