"""Host-side logic of the library compiled with g++ and run on the CPU.

* bph_device_scope.h: every entry point makes its context's device current
  and puts the caller's current device back (a Fortran host that drives
  other work on another GPU from the same thread must not find its device
  switched).  The guard's logic runs here against a fake runtime.
* bph_noalloc_plan.h: the scratch sizing of the allocation-free contraction
  (rejection beyond the 8 MiB array, split-count clamps), including limits
  no constructible context on one GPU reaches.
* bph_slices.h: the zone slices of the split-K tensor-core contraction
  cover every interior zone exactly once for every slice count and chunk
  length (a chunk that read into the next slice would add those zones
  twice).
* bph_compact.h: the compact Green-table layout (symmetric tiles of the
  top and bottom rows, sliding U/V windows of the side rows) contracted
  with the kernel's index arithmetic equals the dense contraction, for
  ragged tile edges, odd radial counts and both symmetry classes.
* bph_direct.h: the closed-form eigenvectors of the vertical second
  difference (reflecting or Dirichlet bottom) are orthonormal and
  diagonalise it, the basis of the direct defect solve; and the solve
  kernel's index arithmetic, emulated lane by lane: the fragment offsets
  follow the m16n8k8 lane layout, the in-place transform over the warp
  tiles equals the dense product with every output written once, the
  residual sweep equals the per-zone FP64 residual bit for bit, and the
  twisted factorization of the radial systems matches an FP64 Thomas solve.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "bipoly_hydro_b200", "csrc")
CPP = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp")


def _run(tmp_path, name):
    exe = tmp_path / name
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", CSRC, os.path.join(CPP, name + ".cpp"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    return out.stdout


def test_device_scope_restores_callers_device(tmp_path):
    assert "all checks passed" in _run(tmp_path, "device_scope_check")


def test_noalloc_plan_limits_and_clamps(tmp_path):
    assert "all checks passed" in _run(tmp_path, "noalloc_plan_check")


def test_zone_slices_cover_each_zone_once(tmp_path):
    assert "all checks passed" in _run(tmp_path, "zone_slice_check")


def test_compact_table_layout_matches_dense_contraction(tmp_path):
    assert "all checks passed" in _run(tmp_path, "compact_layout_check")


def test_vertical_eigen_decomposition(tmp_path):
    assert "all checks passed" in _run(tmp_path, "direct_eigen_check")


def test_library_selects_devices_only_through_the_scope():
    """No source file of the library calls cudaSetDevice except the scope
    header, so no entry point can leave the caller on another device."""
    offenders = []
    for name in sorted(os.listdir(CSRC)):
        if not name.endswith((".cu", ".cuh", ".h")) or name == "bph_device_scope.h":
            continue
        text = open(os.path.join(CSRC, name)).read()
        for m in re.finditer(r"cudaSetDevice\s*\(", text):
            offenders.append(f"{name}:{text[:m.start()].count(chr(10)) + 1}")
    assert not offenders, offenders


def test_direct_kernel_index_arithmetic(tmp_path):
    out = _run(tmp_path, "direct_tiles_check")
    assert "all checks passed" in out
    assert "nr 128 nz  96: cpb 8, 102400 bytes" in out
