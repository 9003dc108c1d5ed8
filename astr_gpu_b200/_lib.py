"""ctypes loader for libastr_b200.so (the sm_100a C ABI declared in include/astr_b200.h).

The library is built in-tree by ``python -m astr_gpu_b200.build``. There is no CPU fallback:
importing a compute entry point without the library raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libastr_b200.so")
# the same C ABI built without multiply-add contraction (-fmad=false), for strict-parity checks
STRICT_LIB_PATH = os.path.join(HERE, "libastr_b200_strict.so")

ASTR_OK, ASTR_ERR_ARG, ASTR_ERR_CUDA, ASTR_ERR_STATE, ASTR_ERR_UNSUPPORTED, ASTR_ERR_NOMEM = 0, -1, -2, -3, -4, -5
ASTR_HOST, ASTR_DEVICE = 0, 1

_vp = ctypes.c_void_p
_pvp = ctypes.POINTER(ctypes.c_void_p)
_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_ip = ctypes.POINTER(ctypes.c_int)
_i = ctypes.c_int
_d = ctypes.c_double


class AstrParams(ctypes.Structure):
    _fields_ = [("im", _i), ("jm", _i), ("km", _i), ("mach", _d), ("reynolds", _d), ("prandtl", _d),
                ("gamma", _d), ("ref_tem", _d), ("sutherland", _d), ("alfa_filter", _d), ("beta_halo", _d),
                ("beta_bound", _d), ("filter_on", _i), ("ntype", _i * 3), ("twall", _d),
                ("conschm", _i), ("bfacmpld", _d), ("lchardecomp", _i), ("shkcrt", _d)]


SIGNATURES = {
    "astr_init": (_i, [_i, _pvp]),
    "astr_destroy": (_i, [_vp]),
    "astr_last_error": (ctypes.c_char_p, [_vp]),
    "astr_set_stream": (_i, [_vp, _vp]),
    "astr_synchronize": (_i, [_vp]),
    "astr_fd_scheme_create": (_i, [_vp, ctypes.c_char_p, _i, _i, _pvp]),
    "astr_filter_create": (_i, [_vp, _i, _i, _d, _d, _d, _i, _pvp]),
    "astr_scheme_destroy": (_i, [_vp]),
    "astr_scheme_ac": (_i, [_vp, _dp, _ip, _ip]),
    "astr_deriv_lines": (_i, [_vp, _vp, _i, _vp, _i64p, _i64p, _vp, _i64p, _i64p, _i, _d, _i]),
    "astr_filter_lines": (_i, [_vp, _vp, _i, _vp, _i64p, _i64p, _vp, _i64p, _i64p, _i, _i]),
    "astr_flux_create": (_i, [_vp, _i, _i, _i, ctypes.c_char, _d, _pvp]),
    "astr_flux_lines": (_i, [_vp, _vp, _i, _vp, _i64p, _i64p, _vp, _i64p, _i64p, _i, _i]),
    "astr_flux_diff_lines": (_i, [_vp, _vp, _i, _vp, _i64p, _i64p, _vp, _i64p, _i64p, _i, _d, _i, _i]),
    "astr_state_create": (_i, [_vp, ctypes.POINTER(AstrParams), _pvp]),
    "astr_state_destroy": (_i, [_vp]),
    "astr_state_init_tgv": (_i, [_vp]),
    "astr_state_upload": (_i, [_vp, _vp, _i64p, _i64p, _i]),
    "astr_state_download": (_i, [_vp, _vp, _i64p, _i64p, _i]),
    "astr_cfl_dt": (_i, [_vp, _d, _dp]),
    "astr_rhs": (_i, [_vp, _vp, _i64p, _i64p, _i]),
    "astr_rk3_step": (_i, [_vp, _d, _i]),
    "astr_rk3_step_host": (_i, [_vp, _vp, _i64p, _i64p, _d, _i, _dp]),
    "astr_history": (_i, [_vp, _dp, _i, _ip]),
    "astr_diagnostics": (_i, [_vp, _dp]),
    "astr_state_use_graph": (_i, [_vp, _i]),
    "astr_state_split_filter": (_i, [_vp, _i]),
    "astr_pass_timings": (_i, [_vp, _d, _i, _dp]),
    "astr_state_autotune": (_i, [_vp, _i]),
    "astr_state_launch_shapes": (_i, [_vp, _ip]),
    "astr_state_set_launch_shape": (_i, [_vp, _i, _i, _i, _i, _i, _i]),
    "astr_ensemble_create": (_i, [_vp, _pvp, _i, _pvp]),
    "astr_ensemble_destroy": (_i, [_vp]),
    "astr_ensemble_step": (_i, [_vp, _dp, _i]),
    "astr_adjoint_create": (_i, [_vp, _i, _pvp]),
    "astr_adjoint_destroy": (_i, [_vp]),
    "astr_adjoint_forward": (_i, [_vp, _d, _i, _dp]),
    "astr_adjoint_backward": (_i, [_vp, _vp, _i64p, _i64p, _i]),
    "astr_step_vjp": (_i, [_vp, _d, _vp, _vp, _i64p, _i64p, _i]),
    "astr_scheme_apply_transpose": (_i, [_vp, _vp, _i, _vp, _i64p, _vp, _i, _d]),
    "astr_cfl_dt_noalloc": (_i, [_vp, _vp, _i64p, _i64p, _i, _i, _i, _d, _d, _d, _dp]),
    "astr_full_create": (_i, [_vp, ctypes.POINTER(AstrParams), _pvp]),
    "astr_full_destroy": (_i, [_vp]),
    "astr_full_upload": (_i, [_vp, _vp, _i64p, _i64p, _i]),
    "astr_full_download": (_i, [_vp, _vp, _i64p, _i64p, _i]),
    "astr_full_step": (_i, [_vp, _d, _i]),
    "astr_full_rhs": (_i, [_vp, _vp, _i64p, _i64p, _i]),
    "astr_full_history": (_i, [_vp, _dp, _i, _ip]),
    "astr_h5io_init": (_i, [ctypes.c_char_p, ctypes.c_char_p, _pvp]),
    "astr_h5io_end": (_i, [_vp]),
    "astr_h5_last_error": (ctypes.c_char_p, [_vp]),
    "astr_h5write_r8": (_i, [_vp, ctypes.c_char_p, _i, _i64p, _vp]),
    "astr_h5write_i4": (_i, [_vp, ctypes.c_char_p, _i, _i64p, _vp]),
    "astr_h5read_r8": (_i, [_vp, ctypes.c_char_p, _i, _i64p, _i64p, ctypes.c_char, _vp]),
    "astr_h5read_i4": (_i, [_vp, ctypes.c_char_p, _i, _i64p, _i64p, ctypes.c_char, _vp]),
    "astr_h5_dataset_info": (_i, [_vp, ctypes.c_char_p, _ip, _i64p, _ip, _ip]),
    "astr_h5_count": (_i, [_vp, _ip]),
    "astr_h5_name": (_i, [_vp, _i, ctypes.c_char_p, _i]),
    "astr_state_write_flowfield": (_i, [_vp, ctypes.c_char_p]),
    "astr_state_read_flowfield": (_i, [_vp, ctypes.c_char_p, ctypes.c_char, _ip, _dp]),
    "astr_full_write_flowfield": (_i, [_vp, ctypes.c_char_p]),
    "astr_full_read_flowfield": (_i, [_vp, ctypes.c_char_p, ctypes.c_char, _ip, _dp]),
}

_libs = {}


def load(strict: bool = False):
    """Load the shared library (no compute happens here; works on a machine without a GPU).
    `strict` loads the variant built with -fmad=false."""
    path = STRICT_LIB_PATH if strict else LIB_PATH
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m astr_gpu_b200.build"
                               f"{' --strict' if strict else ''}`")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _libs[path] = L
    return _libs[path]
