"""C-ABI checks that need no GPU: the library loads and exports every declared entry point."""
import ctypes
import os
import subprocess

import pytest

import crmpm_b200 as cb


def test_library_builds_and_loads():
    cb.build_library()
    assert os.path.exists(cb.LIB_PATH)
    L = cb.lib()
    assert L.CrB200GetVersion() == 100


def test_every_declared_symbol_is_exported():
    declared = cb.declared_symbols()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", cb.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    # nothing beyond the declared C ABI leaks out of the library
    extra = sorted(s for s in exported if s.startswith("CrB200") and s not in declared)
    assert not extra, extra


def test_create_rejects_bad_arguments_without_gpu():
    L = cb.lib()
    h = ctypes.c_void_p()
    mn = (ctypes.c_float * 3)(0, 0, 0)
    mx = (ctypes.c_float * 3)(1, 1, 1)
    # CPU solver kinds have no counterpart here
    assert L.CrB200SolverCreate(0, 10, ctypes.c_float(0.1), mn, mx, None, ctypes.byref(h)) == -3
    assert b"GPU solver types" in L.CrB200GetLastError()
    assert L.CrB200SolverCreate(1, 0, ctypes.c_float(0.1), mn, mx, None, ctypes.byref(h)) == -1
    assert L.CrB200SolverCreate(1, 10, ctypes.c_float(-1.0), mn, mx, None, ctypes.byref(h)) == -1
    assert L.CrB200SolverCreate(1, 10, ctypes.c_float(0.5), mn, mx, None, ctypes.byref(h)) == -1  # < 5 nodes
    assert L.CrB200SolverRelease(None) == -1


def test_grid_dims_match_reference_formula():
    from crmpm_b200 import scenes

    L = cb.lib()
    for sc in (scenes.cube_drop(), scenes.tissue_slab(size=(0.2, 0.1, 0.2)), scenes.pb_cutting(size=(0.1, 0.05, 0.1))):
        s = cb.GpuSolver(sc.solver_type, 16, sc.cell_size, sc.grid_min, sc.grid_max)
        assert s.grid_dims() == sc.grid_dims()
        s.release()
