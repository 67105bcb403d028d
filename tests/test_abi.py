"""The C-ABI library: builds for sm_100a, loads, exports every declared
symbol, validates arguments on the host (CPU; no kernel is launched)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from leviathan_v1_b200 import _build, _lib

HEADER = os.path.join(_build.REPO_DIR, "include", "leviathan_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:lev|leviathan)_[a-z0-9_]+)\s*\(", src)))


def test_library_builds_and_loads():
    path = _build.build()
    assert os.path.exists(path)
    lib = _lib.load()
    assert lib.lev_version().decode().startswith("leviathan_b200")


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and every one has a ctypes prototype in the binding
    assert set(names) <= set(_lib.PROTOTYPES), set(names) - set(_lib.PROTOTYPES)


def test_reference_abi_symbols_present():
    """The ten entry points of the reference (leviathan_kernel.cu:270-497)."""
    lib = _lib.load()
    for n in ("leviathan_init", "leviathan_step", "leviathan_get_theta",
              "leviathan_set_theta", "leviathan_free", "leviathan_set_gain",
              "leviathan_get_gain", "leviathan_set_gain_controller",
              "leviathan_get_vram_usage", "leviathan_reset_weights"):
        assert hasattr(lib, n)


def test_default_params_are_reference_constants():
    p = _lib.default_params().to_dict()
    want = dict(eta=0.01, lam=0.001, gamma=0.05, alpha_eps=0.1, kappa_w=0.01,
                w_min=0.0, w_max=2.0, g=1.5, r0=0.5, beta=0.01, mu=0.01,
                g_rest=1.5, g_min=0.1, g_max=5.0, gain_controller=1)
    for k, v in want.items():
        assert p[k] == np.float32(v), k
    assert C.sizeof(_lib.LevParams) == 64


def _tiny():
    rp = np.array([0, 1, 2], np.int32)
    col = np.array([1, 0], np.int32)
    d = np.array([1, 1], np.uint8)
    w = np.array([0.5, 0.5], np.float32)
    th = np.array([0.1, 0.2], np.float32)
    om = np.array([1.0, 1.0], np.float32)
    return rp, col, d, w, th, om


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("N,max_delay,rp_fix,msg", [
    (0, 5, None, "N must be"),
    (2, 256, None, "max_delay"),
    (2, -1, None, "max_delay"),
    (2, 5, np.array([1, 1, 2], np.int32), "row_ptr[0]"),
    (2, 5, np.array([0, 1, -1], np.int32), "row_ptr[N] is negative"),
])
def test_create_rejects_bad_arguments_before_any_device_work(N, max_delay, rp_fix, msg):
    """Scalar arguments and the ends of row_ptr.  A decreasing row_ptr is
    found by the layout pass, which runs while the edge arrays are uploaded
    (test_engine_gpu.py::test_invalid_row_ptr_and_sizes_rejected)."""
    lib = _lib.load()
    rp, col, d, w, th, om = _tiny()
    if rp_fix is not None:
        rp = rp_fix
    h = C.c_void_p()
    rc = lib.lev_create(C.byref(h), N, max_delay, _ptr(rp), _ptr(col), _ptr(d),
                        _ptr(w), _ptr(th), _ptr(th), _ptr(om), None, 0)
    assert rc == _lib.LEV_ERR_ARG
    assert msg in lib.lev_last_error().decode()
    assert not h.value


def test_bad_math_mode_and_params():
    lib = _lib.load()
    rp, col, d, w, th, om = _tiny()
    h = C.c_void_p()
    rc = lib.lev_create(C.byref(h), 2, 3, _ptr(rp), _ptr(col), _ptr(d), _ptr(w),
                        _ptr(th), _ptr(th), _ptr(om), None, 7)
    assert rc == _lib.LEV_ERR_ARG
    p = _lib.make_params(w_min=3.0, w_max=1.0)
    rc = lib.lev_create(C.byref(h), 2, 3, _ptr(rp), _ptr(col), _ptr(d), _ptr(w),
                        _ptr(th), _ptr(th), _ptr(om), C.byref(p), 0)
    assert rc == _lib.LEV_ERR_ARG and "w_min" in lib.lev_last_error().decode()


def test_reference_abi_init_returns_null_instead_of_exiting():
    lib = _lib.load()
    rp, col, d, w, th, om = _tiny()
    h = lib.leviathan_init(0, 5, _ptr(rp), _ptr(col), _ptr(d), _ptr(w), _ptr(th),
                           _ptr(th), _ptr(om))
    assert not h
    # step on a null handle reports and returns NaN
    assert np.isnan(lib.leviathan_step(None, C.c_float(0.05)))


def test_null_handle_calls_are_errors():
    lib = _lib.load()
    assert lib.lev_step(None, C.c_float(0.05), None) == _lib.LEV_ERR_ARG
    assert lib.lev_step_n(None, C.c_float(0.05), 3, None) == _lib.LEV_ERR_ARG
    assert lib.lev_destroy(None) == _lib.LEV_OK
    el = C.c_int32()
    assert lib.lev_part_pairs(None, C.byref(el)) == _lib.LEV_ERR_ARG
    buf = C.c_void_p(16)  # never dereferenced: the handle check comes first
    assert lib.lev_part_pair_begin(None, C.c_float(0.05), buf) == _lib.LEV_ERR_ARG
    assert lib.lev_part_pair_finish(None, C.c_float(0.05), buf) == _lib.LEV_ERR_ARG


def test_python_engine_validates_sizes():
    from leviathan_v1_b200 import LeviathanEngine

    rp, col, d, w, th, om = _tiny()
    with pytest.raises(ValueError, match="row_ptr"):
        LeviathanEngine(3, 5, rp, col, d, w, th, th, om)
    with pytest.raises(ValueError, match="weights"):
        LeviathanEngine(2, 5, rp, col, d, w[:1], th, th, om)
    with pytest.raises(ValueError, match="theta"):
        LeviathanEngine(2, 5, rp, col, d, w, th[:1], th, om)


def test_sm100a_only_build_flags():
    assert "arch=compute_100a,code=sm_100a" in " ".join(_build.ARCH_FLAGS)
    assert "--use_fast_math" not in _build.NVCC_FLAGS
