"""The C ABI library loads and exports every symbol include/bph.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "bph.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"\b(bph_[a-z_]+)\s*\(", text)


def test_header_declares_the_mirrored_symbols(bph):
    syms = declared_symbols()
    assert len(syms) == len(set(syms))
    assert set(syms) == set(bph.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol(bph):
    lib = ctypes.CDLL(bph.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_string(bph):
    assert "sm_100a" in bph.version()


@pytest.mark.parametrize("grid,msg", [
    ((4, 10, 16, 0.1, 2, 4), "numr"),
    ((10, 10, 24, 0.1, 2, 4), "power of two"),
    ((10, 10, 1024, 0.1, 2, 4), "power of two"),
    ((10, 10, 16, 0.1, 4, 4), "isym"),
    ((10, 10, 16, 0.1, 2, 1), "mmax"),
    ((10, 10, 64, 0.1, 2, 40), "too small"),
    ((10, 10, 64, 0.1, 3, 20), "too small"),
    ((10, 10, 16, -0.1, 2, 4), "dr"),
])
def test_invalid_grids_are_rejected_before_any_device_work(bph, grid, msg):
    with pytest.raises(bph.BphError) as ei:
        bph.PotentialSolver(*grid)
    assert ei.value.code == bph.BPH_ERR_INVALID
    assert msg in str(ei.value)


def test_null_context_is_an_error(bph):
    lib = bph.load_library()
    assert lib.bph_potential_solver(None, None, None, 0) == bph.BPH_ERR_INVALID
    assert lib.bph_destroy(None) == bph.BPH_OK


def test_host_registration_rejects_bad_arguments_before_device_work(bph):
    lib = bph.load_library()
    assert lib.bph_register_host(None, 1024) == bph.BPH_ERR_INVALID
    buf = ctypes.create_string_buffer(64)
    assert lib.bph_register_host(ctypes.cast(buf, ctypes.c_void_p), 0) == bph.BPH_ERR_INVALID
    assert lib.bph_unregister_host(None) == bph.BPH_ERR_INVALID


def test_product_does_not_import_the_oracle():
    """The product package never imports, links or loads the CPU oracle."""
    pkg = os.path.join(ROOT, "bipoly_hydro_b200")
    bad = re.compile(r"(import\s+oracle|from\s+oracle|liborc|bph_oracle|orc_[a-z])")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp", "Makefile")):
                src = open(os.path.join(dirpath, f)).read()
                assert not bad.search(src), f


def test_null_handles_of_batches_plans_and_servers_are_errors(bph):
    """The batch, plan and server entry points reject NULL handles and bad
    counts before any device work."""
    import ctypes

    lib = bph.load_library()
    inv = bph.BPH_ERR_INVALID
    assert lib.bph_batch_solve(None, 1, None, None, 0, 0) == inv
    assert lib.bph_batch_solve_converged(None, 1, None, None, 10, 1, 1e-11, 10, 0, 0, None, None) == inv
    assert lib.bph_batch_destroy(None) == bph.BPH_OK
    out = ctypes.c_void_p(123)
    assert lib.bph_plan_create(0, None, None, None, None, ctypes.byref(out)) == inv
    assert out.value is None  # cleared on failure
    assert lib.bph_plan_launch(None, 2, None) == inv
    assert lib.bph_plan_synchronize(None, None) == inv
    assert lib.bph_plan_launches(None) == 0
    assert lib.bph_plan_destroy(None) == bph.BPH_OK
    assert lib.bph_server_set_converged(None, 10, 1e-11, 10, 0) == inv
    assert lib.bph_server_destroy(None) in (bph.BPH_OK, inv)


def test_info_keys_follow_the_header(bph):
    """PotentialSolver.info() names every BPH_INFO_* index of include/bph.h,
    in order, and the mixed kinds and contraction kinds match their defines."""
    import os
    import re

    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "bph.h")).read()
    defs = {int(v): k.lower() for k, v in re.findall(r"#define BPH_INFO_([A-Z0-9_]+) (\d+)", hdr)}
    assert sorted(defs) == list(range(len(defs)))
    assert tuple(defs[i] for i in range(len(defs))) == bph.solver.INFO_KEYS
    kinds = dict(re.findall(r"#define (BPH_MIXED_[A-Z_]+|BPH_CONTRACT_[A-Z]+) (\d+)", hdr))
    S = bph.solver
    assert int(kinds["BPH_MIXED_ADI_WARP"]) == S.MIXED_ADI_WARP
    assert int(kinds["BPH_MIXED_DIRECT"]) == S.MIXED_DIRECT
    assert int(kinds["BPH_CONTRACT_COMPACT"]) == S.CONTRACT_COMPACT and int(kinds["BPH_CONTRACT_FULL"]) == S.CONTRACT_FULL
