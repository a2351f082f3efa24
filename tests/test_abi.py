"""The C-ABI library loads without a GPU and exports every declared entry point."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from twophaseflow_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms |= set(re.findall(r"\b(tpf_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "tpf_ccd_apply" in syms and "tpf_ppe_solve" in syms


def test_library_loads_and_exports_all_symbols():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.fail("libtpf.so is not built (python -m twophaseflow_b200.build)")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"missing exports: {missing}"


def test_python_binding_covers_header():
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_host_only_calls_without_gpu():
    lib = _lib.load()
    assert lib.tpf_version() >= 10000
    # the launch autotuner's switch and counter need no device
    assert lib.tpf_launch_autotune_entries() >= 0
    assert lib.tpf_set_launch_autotune(1) == _lib.TPF_OK
    assert lib.tpf_set_launch_autotune(-1) == _lib.TPF_EINVAL
    o = _lib.tpf_ppe_options()
    lib.tpf_ppe_default_options(ctypes.byref(o))
    # reference defaults (fvm_matrixfree.py:90-127)
    assert o.method == _lib.TPF_PPE_GMRES and o.precond == _lib.TPF_PRECOND_LINE
    assert o.tol == 1e-8 and o.maxiter == 500 and o.restart == 80 and o.c_tau == 2.0 and o.pcr_stages == 4
    # the learned solver's defaults: flexible GMRES(60), 16 sweeps at 0.8, PCG fallback
    lo = _lib.tpf_learned_options()
    lib.tpf_lppe_default_options(ctypes.byref(lo))
    assert lo.outer == 1 and lo.restart == 60 and lo.smooth == 16 and lo.omega == 0.8 and lo.fallback == 1
    assert lo.tol == 1e-8 and lo.stall_checks == 16 and lo.check_every == 8 and lo.stall_factor == 0.5


def test_invalid_arguments_fail_closed_on_host():
    lib = _lib.load()
    h = ctypes.c_void_p()
    # wall closure needs n_pts >= 6 (ccd_solver.py:459-465) -> ValueError
    st = lib.tpf_ccd_plan_create(ctypes.byref(h), 5, 0.25, _lib.TPF_BC_WALL, _lib.TPF_F64)
    assert st == _lib.TPF_EINVAL
    assert "n_pts >= 6" in _lib.last_error()
    with pytest.raises(ValueError, match="n_pts >= 6"):
        _lib.check(st)
    st = lib.tpf_ccd_plan_create(ctypes.byref(h), 3, 0.25, _lib.TPF_BC_PERIODIC, _lib.TPF_F64)
    assert st == _lib.TPF_EINVAL
    o = _lib.tpf_ppe_options()
    lib.tpf_ppe_default_options(ctypes.byref(o))
    o.method = _lib.TPF_PPE_CG
    o.precond = _lib.TPF_PRECOND_LINE
    N = (ctypes.c_int64 * 2)(4, 4)
    st = lib.tpf_ppe_create(ctypes.byref(h), 2, N, None, 12, ctypes.byref(o))
    assert st == _lib.TPF_EINVAL
