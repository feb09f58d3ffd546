"""ctypes binding of libekpnp.so (C ABI declared in include/ekpnp.h).

The shared library is built in-tree by ek-pnp_b200/build.py.  There is no
fallback: if the library is missing or cannot be loaded this module raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libekpnp.so")

EK_OK = 0
EK_ERR_INVALID = 1
EK_ERR_CUDA = 2
EK_ERR_NOMEM = 3
EK_ERR_NAN = 4
EK_ERR_TIMEOUT = 5
EK_ERR_UNSUPPORTED = 6
EK_ERR_TOO_LARGE = 7

STORE_F64, STORE_F32, STORE_F16 = 0, 1, 2
FLAG_FORCE, FLAG_REST_QUIRK, FLAG_MOMENTS_EVERY_STEP, FLAG_EXPLICIT_E = 1, 2, 4, 8

_DOUBLE_FIELDS = ("dx", "dy", "dt", "cfl", "cs2", "lx", "rho0", "c0", "nu", "magic_f", "diff_p",
                  "magic_p", "mob_p", "diff_n", "magic_n", "mob_n", "eps", "f_charge", "zeta_lo",
                  "zeta_hi", "cp_lo", "cp_hi", "cn_lo", "cn_hi", "ext_x", "exf", "uw")


class EkParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("storage", ctypes.c_int32),
                ("flags", ctypes.c_int32)] + [(n, ctypes.c_double) for n in _DOUBLE_FIELDS]

    @classmethod
    def from_dict(cls, d):
        p = cls()
        for name, _ in cls._fields_:
            if name not in d:
                raise KeyError(f"parameter '{name}' missing")
            setattr(p, name, d[name])
        return p

    def to_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class EkError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"libekpnp status {status}: {message}")
        self.status = status


_lib = None

_P = ctypes.POINTER
_dp = _P(ctypes.c_double)
_fp = _P(ctypes.c_float)
_SIGS = {
    "ek_version": ([], ctypes.c_int),
    "ek_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "ek_last_error": ([], ctypes.c_char_p),
    "ek_set_device": ([ctypes.c_int32], ctypes.c_int),
    "ek_get_device_count": ([_P(ctypes.c_int32)], ctypes.c_int),
    "ek_params_default": ([_P(EkParams), ctypes.c_int32, ctypes.c_int32], ctypes.c_int),
    "ek_create": ([_P(EkParams), _P(ctypes.c_void_p)], ctypes.c_int),
    "ek_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "ek_set_stream": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "ek_get_params": ([ctypes.c_void_p, _P(EkParams)], ctypes.c_int),
    "ek_set_fields": ([ctypes.c_void_p] + [_dp] * 8, ctypes.c_int),
    "ek_set_fields_device": ([ctypes.c_void_p] + [ctypes.c_void_p] * 8, ctypes.c_int),
    "ek_mlp_set_wait_cycles": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "ek_wait_selftest": ([ctypes.c_int64, ctypes.c_int32], ctypes.c_int),
    "ek_set_wall_profile": ([ctypes.c_void_p] + [_dp] * 6, ctypes.c_int),
    "ek_init_equilibrium": ([ctypes.c_void_p], ctypes.c_int),
    "ek_tile_x": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "ek_step": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "ek_poisson": ([ctypes.c_void_p], ctypes.c_int),
    "ek_poisson_jacobi": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                           _P(ctypes.c_int32), _dp], ctypes.c_int),
    "ek_get_fields": ([ctypes.c_void_p] + [_dp] * 8, ctypes.c_int),
    "ek_get_fields_device": ([ctypes.c_void_p] + [ctypes.c_void_p] * 8, ctypes.c_int),
    "ek_residual": ([ctypes.c_void_p, ctypes.c_int32, _dp], ctypes.c_int),
    "ek_step_count": ([ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_sync": ([ctypes.c_void_p], ctypes.c_int),
    "ek_field_pointers": ([ctypes.c_void_p, _P(ctypes.c_void_p), _P(ctypes.c_int32)], ctypes.c_int),
    "ek_profile_enable": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "ek_profile_read": ([ctypes.c_void_p, _dp, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_mark": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "ek_elapsed": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, _dp], ctypes.c_int),
    "ek_launch_count": ([ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_poisson_noalloc": ([_P(EkParams)] + [ctypes.c_void_p] * 6, ctypes.c_int),
    "ek_rebase": ([ctypes.c_void_p], ctypes.c_int),
    "ek_set_option": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64], ctypes.c_int),
    "ek_set_rebase_interval": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "ek_init_poisson_boltzmann": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                   ctypes.c_double], ctypes.c_int),
    "ek_batch_create": ([ctypes.c_void_p, ctypes.c_int32, _P(ctypes.c_void_p)], ctypes.c_int),
    "ek_batch_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "ek_batch_count": ([ctypes.c_void_p, _P(ctypes.c_int32), _P(ctypes.c_int64)], ctypes.c_int),
    "ek_batch_channel": ([ctypes.c_void_p, ctypes.c_int32, _P(ctypes.c_void_p)], ctypes.c_int),
    "ek_batch_stream": ([ctypes.c_void_p, _P(ctypes.c_void_p)], ctypes.c_int),
    "ek_batch_set_cycle": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32], ctypes.c_int),
    "ek_batch_init_equilibrium": ([ctypes.c_void_p], ctypes.c_int),
    "ek_batch_step": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "ek_batch_sync": ([ctypes.c_void_p], ctypes.c_int),
    "ek_batch_step_count": ([ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_batch_launch_count": ([ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_batch_shape_info": ([ctypes.c_int32, _P(ctypes.c_int32), _P(ctypes.c_int32), _P(ctypes.c_int32)],
                            ctypes.c_int),
    "ek_batch_shape": ([ctypes.c_void_p, _P(ctypes.c_int32)], ctypes.c_int),
    "ek_batch_set_shape": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "ek_batch_autotune": ([ctypes.c_void_p, ctypes.c_int32, _P(ctypes.c_int32), _dp], ctypes.c_int),
    "ek_batch_residual": ([ctypes.c_void_p, ctypes.c_int32, _dp, _dp], ctypes.c_int),
    "ek_batch_set_active": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "ek_batch_resync": ([ctypes.c_void_p], ctypes.c_int),
    "ek_batch_restart": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "ek_batch_active": ([ctypes.c_void_p, ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_write_restart": ([ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double] + [_dp] * 8, ctypes.c_int),
    "ek_read_restart": ([ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, _dp] + [_dp] * 8, ctypes.c_int),
    "ek_save_restart": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double], ctypes.c_int),
    "ek_load_restart": ([ctypes.c_void_p, ctypes.c_char_p, _dp], ctypes.c_int),
    "ek_write_tecplot": ([ctypes.c_char_p, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                          ctypes.c_double, ctypes.c_double] + [_dp] * 8, ctypes.c_int),
    "ek_write_dmd": ([ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _dp], ctypes.c_int),
    "ek_diag_current": ([ctypes.c_int32, ctypes.c_int32, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp],
                        ctypes.c_int),
    "ek_diag_umax": ([ctypes.c_int32, ctypes.c_int32, _dp, _dp], ctypes.c_int),
    "ek_mlp_create": ([ctypes.c_int32, ctypes.c_uint64, _P(ctypes.c_void_p)], ctypes.c_int),
    "ek_mlp_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "ek_mlp_param_count": ([ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_mlp_get_params": ([ctypes.c_void_p, _fp], ctypes.c_int),
    "ek_mlp_set_params": ([ctypes.c_void_p, _fp], ctypes.c_int),
    "ek_mlp_set_data": ([ctypes.c_void_p, _fp, _fp, ctypes.c_int64], ctypes.c_int),
    "ek_mlp_train": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_float, _dp], ctypes.c_int),
    "ek_mlp_gradients": ([ctypes.c_void_p, _fp, _fp, _fp, _dp], ctypes.c_int),
    "ek_mlp_forward": ([ctypes.c_void_p, _fp, ctypes.c_int64, _fp], ctypes.c_int),
    "ek_mlp_launch_count": ([ctypes.c_void_p, _P(ctypes.c_int64)], ctypes.c_int),
    "ek_gemm_bf16": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p], ctypes.c_int),
}


def lib():
    """Load libekpnp.so once and declare every exported signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python ek-pnp_b200/build.py`")
        h = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(h, name)
            fn.argtypes = args
            fn.restype = res
        _lib = h
    return _lib


def check(rc):
    if rc != EK_OK:
        msg = lib().ek_last_error().decode(errors="replace")
        raise EkError(rc, msg or lib().ek_status_string(rc).decode())
    return rc


def exported_symbols():
    return list(_SIGS)
