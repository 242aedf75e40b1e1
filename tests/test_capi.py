"""The C-ABI library loads and exports every entry point include/fvm2d.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fvm2d.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fvm2d_\w+)\s*\(", text)))


def test_header_declares_the_solver_api():
    syms = declared_symbols()
    for must in ("fvm2d_create", "fvm2d_destroy", "fvm2d_solve", "fvm2d_set_state", "fvm2d_get_state",
                 "fvm2d_set_ghost_strategy", "fvm2d_get_computation_time_ms", "fvm2d_get_time_stages_count"):
        assert must in syms


def test_library_exports_every_declared_symbol(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_the_header(pkg):
    from importlib import import_module
    sigs = {n for n, _, _ in import_module("2d_fvm_cuda_b200._lib").SIGNATURES}
    assert set(declared_symbols()) <= sigs


def test_bad_arguments_fail_cleanly_without_a_device(pkg):
    lib = pkg.load()
    h = ctypes.c_void_p()
    assert lib.fvm2d_create(ctypes.byref(h), 4, 100) == 1
    assert b"at least 6" in lib.fvm2d_last_error()
    assert lib.fvm2d_set_cfl(None, 0.5) == 1
    out = (ctypes.c_double * 4)()
    assert lib.fvm2d_get_conserved_totals(None, out) == 1
    assert lib.fvm2d_destroy(None) == 0


def test_create_reports_missing_gpu(pkg):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    lib = pkg.load()
    h = ctypes.c_void_p()
    assert lib.fvm2d_create(ctypes.byref(h), 64, 64) == 2
    assert lib.fvm2d_last_error()


def test_python_mirror_totals_need_a_result(pkg):
    s = pkg.RGRP_2D_CUDA()
    with pytest.raises(RuntimeError):
        s.getConservedTotals()
