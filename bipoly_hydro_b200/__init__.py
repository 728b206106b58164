"""B200-native self-gravity Poisson solve of bipoly_hydro (potsetup + potential_solver).

The solver runs in ``libbph.so`` (CUDA for sm_100a) behind the C ABI of
``include/bph.h``; this package is its Python host mirror.
"""
from .solver import (  # noqa: F401
    BPH_ERR_CUDA,
    BPH_ERR_INVALID,
    BPH_ERR_NOMEM,
    BPH_ERR_NONFINITE,
    BPH_ERR_STATE,
    BPH_ERR_TIMEOUT,
    BPH_OK,
    EXPORTED_SYMBOLS,
    LIB_PATH,
    BphError,
    Grid,
    PotentialSolver,
    Batch,
    Plan,
    Server,
    load_library,
    read_continuation,
    register_host,
    unregister_host,
    version,
)

__all__ = [
    "PotentialSolver", "Batch", "Plan", "Server", "Grid", "BphError", "load_library", "read_continuation", "register_host",
    "unregister_host", "version", "LIB_PATH", "EXPORTED_SYMBOLS",
    "BPH_OK", "BPH_ERR_INVALID", "BPH_ERR_NOMEM", "BPH_ERR_NONFINITE", "BPH_ERR_CUDA", "BPH_ERR_TIMEOUT",
    "BPH_ERR_STATE",
]
