"""ctypes binding of ``libleviathan_b200.so`` (the C ABI in
``include/leviathan_b200.h``).

The library is built in-tree by ``leviathan_v1_b200._build``.  There is no
fallback: if the library is missing, importing the engine fails loudly.
"""

from __future__ import annotations

import ctypes as C
import os

from . import _build

LEV_OK = 0
LEV_ERR_ARG = -1
LEV_ERR_CUDA = -2
LEV_ERR_STATE = -3
LEV_ERR_NOMEM = -4

LEV_MATH_REFERENCE = 0
LEV_MATH_ACCURATE = 1


class LevParams(C.Structure):
    """Mirror of ``LevParams`` (include/leviathan_b200.h)."""

    _fields_ = [
        ("eta", C.c_float),
        ("lam", C.c_float),
        ("gamma", C.c_float),
        ("alpha_eps", C.c_float),
        ("kappa_w", C.c_float),
        ("w_min", C.c_float),
        ("w_max", C.c_float),
        ("g", C.c_float),
        ("r0", C.c_float),
        ("beta", C.c_float),
        ("mu", C.c_float),
        ("g_rest", C.c_float),
        ("g_min", C.c_float),
        ("g_max", C.c_float),
        ("gain_controller", C.c_int32),
        ("reserved", C.c_int32),
    ]

    FIELDS = ("eta", "lam", "gamma", "alpha_eps", "kappa_w", "w_min", "w_max",
              "g", "r0", "beta", "mu", "g_rest", "g_min", "g_max",
              "gain_controller")

    def to_dict(self) -> dict:
        return {k: (int(getattr(self, k)) if k == "gain_controller"
                    else float(getattr(self, k))) for k in self.FIELDS}


_P = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_f32 = C.c_float

# name -> (restype, argtypes)
PROTOTYPES = {
    "lev_last_error": (C.c_char_p, []),
    "lev_version": (C.c_char_p, []),
    "lev_default_params": (None, [C.POINTER(LevParams)]),
    "lev_create": (C.c_int, [C.POINTER(_P), _i32, _i32, _P, _P, _P, _P, _P, _P,
                             _P, C.POINTER(LevParams), _i32]),
    "lev_batch_create": (C.c_int, [C.POINTER(_P), _i32, _P, _P, _P, _P, _P, _P,
                                   _P, _P, _P, C.POINTER(LevParams), _i32]),
    "lev_destroy": (C.c_int, [_P]),
    "lev_create_profile": (C.c_int, [_P, _P]),
    "lev_trim_memory": (C.c_int, []),
    "lev_num_nets": (C.c_int, [_P, C.POINTER(_i32)]),
    "lev_total_nodes": (C.c_int, [_P, C.POINTER(_i64)]),
    "lev_total_edges": (C.c_int, [_P, C.POINTER(_i64)]),
    "lev_net_shape": (C.c_int, [_P, _i32, C.POINTER(_i32), C.POINTER(_i64),
                                C.POINTER(_i32)]),
    "lev_step": (C.c_int, [_P, _f32, _P]),
    "lev_step_n": (C.c_int, [_P, _f32, _i32, _P]),
    "lev_step_n_async": (C.c_int, [_P, _f32, _i32]),
    "lev_sync": (C.c_int, [_P]),
    "lev_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "lev_get_theta": (C.c_int, [_P, _P]),
    "lev_set_theta": (C.c_int, [_P, _P]),
    "lev_get_theta_net": (C.c_int, [_P, _i32, _P]),
    "lev_set_theta_net": (C.c_int, [_P, _i32, _P]),
    "lev_get_weights": (C.c_int, [_P, _P]),
    "lev_reset_weights": (C.c_int, [_P, _P]),
    "lev_get_predictor": (C.c_int, [_P, _P, _P]),
    "lev_set_predictor": (C.c_int, [_P, _P, _P]),
    "lev_get_omega": (C.c_int, [_P, _P]),
    "lev_set_omega": (C.c_int, [_P, _P]),
    "lev_get_ring": (C.c_int, [_P, _i32, _P, C.POINTER(_i32)]),
    "lev_set_ring": (C.c_int, [_P, _i32, _P, _i32]),
    "lev_get_step_count": (C.c_int, [_P, _i32, C.POINTER(_i64)]),
    "lev_set_gain": (C.c_int, [_P, _i32, _f32]),
    "lev_get_gain": (C.c_int, [_P, _i32, C.POINTER(_f32)]),
    "lev_get_r": (C.c_int, [_P, _i32, C.POINTER(_f32)]),
    "lev_set_gain_controller": (C.c_int, [_P, _i32, _i32]),
    "lev_set_params": (C.c_int, [_P, _i32, C.POINTER(LevParams)]),
    "lev_get_params": (C.c_int, [_P, _i32, C.POINTER(LevParams)]),
    "lev_set_math_mode": (C.c_int, [_P, _i32]),
    "lev_get_vram_usage": (C.c_int, [_P, C.POINTER(C.c_size_t)]),
    "lev_cluster_info": (C.c_int, [_P, C.POINTER(_i32), C.POINTER(_i32),
                                   C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i64)]),
    "lev_set_cluster_mode": (C.c_int, [_P, _i32]),
    "lev_grid_info": (C.c_int, [_P, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32),
                                C.POINTER(_i32), C.POINTER(_i64), C.POINTER(_i32)]),
    "lev_set_grid_mode": (C.c_int, [_P, _i32, _i32]),
    "lev_num_pair_variants": (C.c_int, []),
    "lev_pair_variant_info": (C.c_int, [_i32, C.POINTER(_i32), C.POINTER(_i32),
                                        C.POINTER(_i32)]),
    "lev_pair_variant_lanes": (C.c_int, [_i32, C.POINTER(_i32)]),
    "lev_pair_info": (C.c_int, [_P, _i32, C.POINTER(_i32), C.POINTER(_i32),
                                C.POINTER(_i32), C.POINTER(_f32), C.POINTER(_f32)]),
    "lev_set_pair_mode": (C.c_int, [_P, _i32]),
    "lev_set_pair_variant": (C.c_int, [_P, _i32, _i32]),
    "lev_time_launches": (C.c_int, [_P, _f32, _i32, _P]),
    "lev_num_variants": (C.c_int, []),
    "lev_variant_info": (C.c_int, [_i32, C.POINTER(_i32), C.POINTER(_i32),
                                   C.POINTER(_i32)]),
    "lev_class_info": (C.c_int, [_P, _i32, C.POINTER(_i32), C.POINTER(_f32),
                                 C.POINTER(_i64), C.POINTER(_i32)]),
    "lev_set_variant": (C.c_int, [_P, _i32, _i32]),
    "lev_autotune": (C.c_int, [_P, _f32, _i32, _P, _P]),
    "lev_adj_create": (C.c_int, [C.POINTER(_P), _P, _i32, _i32]),
    "lev_adj_destroy": (C.c_int, [_P]),
    "lev_adj_bytes": (C.c_int, [_P, C.POINTER(C.c_size_t)]),
    "lev_adj_forward": (C.c_int, [_P, _f32, _i32, _P, _P, _P, _P, _P, _P]),
    "lev_adj_backward": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "lev_adj_grad_theta0": (C.c_int, [_P, _P]),
    "lev_adj_set_reservoir": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "lev_adj_set_reservoir_grads": (C.c_int, [_P, _P, _P, _P, _P]),
    "lev_adj_grid_info": (C.c_int, [_P, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32),
                                    C.POINTER(_i32), C.POINTER(_i32)]),
    "lev_adj_set_grid_mode": (C.c_int, [_P, _i32, _i32]),
    "lev_adj_set_grid_pairing": (C.c_int, [_P, _i32]),
    "lev_adj_set_grid_wait": (C.c_int, [_P, C.c_uint64, C.c_uint32]),
    "lev_set_grid_wait": (C.c_int, [_P, C.c_uint64, C.c_uint32]),
    "lev_selftest_wraps":(C.c_int, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "lev_step_noalloc":(C.c_int, [_i32, _i32, _i64, _P, _P, _P, _P, _P, _P, _P,
                                   _P, _P, _P, _P, C.POINTER(LevParams), _f32,
                                   _i32, _P]),
    "lev_part_create": (C.c_int, [C.POINTER(_P), _i32, _i32, _i32, _P, _P, _P, _P, _P,
                                  _P, _P, _P, _i32, _i32, _i32, C.POINTER(LevParams),
                                  _i32]),
    "lev_part_info": (C.c_int, [_P, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32),
                                C.POINTER(_i32)]),
    "lev_part_step_begin": (C.c_int, [_P, _f32, _P]),
    "lev_part_step_end": (C.c_int, [_P, _f32, _P, _P]),
    "lev_part_pack": (C.c_int, [_P, _P, _i32, _P]),
    "lev_part_pairs": (C.c_int, [_P, C.POINTER(_i32)]),
    "lev_part_pair_begin": (C.c_int, [_P, _f32, _P]),
    "lev_part_pair_finish": (C.c_int, [_P, _f32, _P]),
    "lev_part_unpack": (C.c_int, [_P, _P, _i32, _P]),
    "lev_part_fill_halo": (C.c_int, [_P, _P]),
    "lev_gen_ws": (C.c_int, [_i32, _i32, C.c_double, C.c_uint64, _i32, _i32, _f32,
                             _f32, _f32, _f32, _P, _P, _P, _P, _P, _P]),
    "lev_hubs_create": (C.c_int, [C.POINTER(_P), _i32, _P]),
    "lev_attach_hubs": (C.c_int, [_P, _i32, _P]),
    "lev_hubs_accumulate": (C.c_int, [_P, _P, _P]),
    "lev_hubs_reset": (C.c_int, [_P]),
    "lev_hubs_read": (C.c_int, [_P, _P, _P, C.POINTER(_i32), C.POINTER(_i64)]),
    "lev_hubs_destroy": (C.c_int, [_P]),
    # reference ABI (leviathan_kernel.cu:21-499)
    "leviathan_init": (_P, [C.c_int, C.c_int, _P, _P, _P, _P, _P, _P, _P]),
    "leviathan_step": (_f32, [_P, _f32]),
    "leviathan_get_theta": (None, [_P, _P]),
    "leviathan_set_theta": (None, [_P, _P]),
    "leviathan_free": (None, [_P]),
    "leviathan_set_gain": (None, [_P, _f32]),
    "leviathan_get_gain": (_f32, [_P]),
    "leviathan_set_gain_controller": (None, [_P, C.c_bool]),
    "leviathan_get_vram_usage": (C.c_size_t, [_P]),
    "leviathan_reset_weights": (None, [_P, _P]),
    "leviathan_engine": (_P, [_P]),
}

_LIB = None


def lib_path() -> str:
    return _build.LIB_PATH


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load the CUDA library (building it in-tree if stale and nvcc exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB_PATH
    if build_if_missing:
        try:
            if _build.needs_build():
                _build.build()
        except RuntimeError:
            if not os.path.exists(path):
                raise
    if not os.path.exists(path):
        raise ImportError(
            f"CUDA library {path} is missing; build it with "
            "`python -m leviathan_v1_b200._build` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class LevError(RuntimeError):
    """Failure reported by the C ABI (status code + message)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def check(rc: int) -> None:
    if rc != LEV_OK:
        msg = load().lev_last_error().decode(errors="replace")
        if rc == LEV_ERR_ARG:
            raise ValueError(msg)
        raise LevError(rc, msg)


def default_params() -> LevParams:
    p = LevParams()
    load().lev_default_params(C.byref(p))
    return p


def make_params(**kw) -> LevParams:
    p = default_params()
    for k, v in kw.items():
        if k not in LevParams.FIELDS:
            raise ValueError(f"unknown parameter {k!r}")
        setattr(p, k, int(v) if k == "gain_controller" else float(v))
    return p
