"""ctypes binding of libedgpu.so (the C ABI declared in include/edgpu.h).

The library is loaded from this package directory. There is no fallback: when the shared
object is missing or fails to load, import raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libedgpu.so")

EDG_OK = 0
EDG_ERR_ARG = -1
EDG_ERR_CUDA = -2
EDG_ERR_NOMEM = -3
EDG_ERR_UNSUPPORTED = -4
EDG_ERR_STATE = -5
EDG_ERR_NOCONV = -6
EDG_ERR_NODEVICE = -8

EDG_FORM_STORED = 0
EDG_FORM_DIRECT = 1
EDG_PREC_F64 = 0
EDG_PREC_F32 = 1
EDG_GS_F64 = 0
EDG_GS_F32_REFINE = 1
EDG_GS_E0_ONLY = 0x100
EDG_LK_F64 = 0
EDG_LK_F32_REFINE = 1

_i = C.c_int
_i64 = C.c_int64
_u64 = C.c_uint64
_d = C.c_double
_p = C.c_void_p
_pd = C.POINTER(C.c_double)
_pf = C.POINTER(C.c_float)
_pi = C.POINTER(C.c_int)
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)
_pp = C.POINTER(C.c_void_p)

# name -> (restype, argtypes); mirrors include/edgpu.h one to one
SIGNATURES = {
    "edg_last_error": (C.c_char_p, []),
    "edg_device_count": (_i, [_pi]),
    "edg_model_create": (_i, [_i, _i, _pd, _pd, _pd, _pd, _d, _d, _i, _i, _pp]),
    "edg_model_destroy": (_i, [_p]),
    "edg_get_sector": (_i, [_i, _i, _i]),
    "edg_get_nup": (_i, [_i, _i]),
    "edg_get_ndw": (_i, [_i, _i]),
    "edg_binomial": (_i64, [_i, _i]),
    "edg_sector_create": (_i, [_p, _i, _i, _i, _pp]),
    "edg_sector_destroy": (_i, [_p]),
    "edg_sector_dims": (_i, [_p, _pi64, _pi64, _pi64]),
    "edg_sector_vlen": (_i, [_p, _pi64]),
    "edg_release_cached_memory": (_i, []),
    "edg_sector_get_maps": (_i, [_p, _pi32, _pi32]),
    "edg_sector_get_hops": (_i, [_p, _i, _pi64, _pi32, _pd, _pi64]),
    "edg_sector_set_stream": (_i, [_p, _p]),
    "edg_sector_release_work": (_i, [_p]),
    "edg_hxv_z": (_i, [_p, _i64, _pd, _pd]),
    "edg_hxv_d": (_i, [_p, _i64, _pd, _pd]),
    "edg_sector_autotune": (_i, [_p, _i, _i, _pd, _pi, _pi]),
    "edg_sector_set_kernels": (_i, [_p, _i, _i]),
    "edg_hxv_dev_f64": (_i, [_p, _p, _p]),
    "edg_hxv_dev_f32": (_i, [_p, _p, _p]),
    "edg_hxv_cols_dev_f64": (_i, [_p, _i64, _i64, _p, _p]),
    "edg_hxv_cols_dev_f32": (_i, [_p, _i64, _i64, _p, _p]),
    "edg_hxv_rows_dev_f64": (_i, [_p, _i64, _i64, _p, _p]),
    "edg_hxv_rows_dev_f32": (_i, [_p, _i64, _i64, _p, _p]),
    "edg_tridiag_d": (_i, [_p, _pd, _i, _d, _i, _pd, _pd, _pd, _pi]),
    "edg_tridiag_dev_f64": (_i, [_p, _p, _i, _d, _i, _pd, _pd, _pd, _pi]),
    "edg_tridiag_dev_f64_noalloc": (_i, [_p, _p, _i, _d, _pd, _pd, _pd, _pi]),
    "edg_ground_state": (_i, [_p, _pd, _u64, _i, _d, _i, _pd, _pd, _pi]),
    "edg_ground_state_keep": (_i, [_p, _pd, _u64, _i, _d, _i, _pd, _pi]),
    "edg_ground_state_stats": (_i, [_p, _pi, _pi]),
    "edg_lowest_k": (_i, [_p, _i, _pd, _u64, _i, _d, _pd, _pd, _pd, _pi]),
    "edg_lowest_k_mode": (_i, [_p, _i, _pd, _u64, _i, _d, _i, _pd, _pd, _pd, _pi]),
    "edg_sector_dense": (_i, [_p, _pd]),
    "edg_sector_dense_dev": (_i, [_p, _p]),
    "edg_state_get": (_i, [_p, _pd]),
    "edg_state_set": (_i, [_p, _pd]),
    "edg_random_vector": (_i, [_u64, _i64, _pd]),
    "edg_apply_cop_dev_f64": (_i, [_p, _p, _i, _i, _i, _d, _i, _p, _p]),
    "edg_apply_diagop_dev_f64": (_i, [_p, _i, _i, _i, _pd, _p, _p]),
    "edg_apply_current_dev_f64": (_i, [_p, _p, _p]),
    "edg_observables": (_i, [_p, _d, _pd, _pd, _pd, _pd, _pd]),
    "edg_energy": (_i, [_p, _d, _pd, _pd, _pd, _pd]),
    "edg_gf_chain": (_i, [_p, _p, _i, _i, _i, _i, _i, _i, _d, _pd, _pd, _pd, _pi]),
    "edg_chi_chain": (_i, [_p, _i, _i, _i, _pd, _i, _i, _d, _pd, _pd, _pd, _pi]),
    "edg_oc_chain": (_i, [_p, _i, _i, _d, _pd, _pd, _pd, _pi]),
    "edg_eval_poles": (_i, [_i64, _pd, _pd, _i64, _pd, _pd, _pd, _pd]),
    "edg_tridiag_block_dev": (_i, [_p, _i, _p, _i, _d, _i, _pd, _pd, _pd, _pi]),
    "edg_tridiag_eigh": (_i, [_i, _pd, _pd, _pd, _pd]),
    "edg_tridiag_lowest": (_i, [_i, _pd, _pd, _i, _pd, _pd]),
    "edg_poles_weights": (_i, [_i, _pd, _pd, _d, _d, _i, _pd, _pd]),
    "edg_gf_chain_block": (_i, [_p, _p, _i, _i, _pi, _pi, _i, _i, _i, _d, _pd, _pd, _pd, _pi]),
    "edg_chi_chain_block": (_i, [_p, _i, _i, _pi, _pi, _pd, _i, _i, _d, _pd, _pd, _pd, _pi]),
    "edg_poles_weights_block": (_i, [_i, _i, _pd, _pd, _pd, _pi, _d, _i, _pd, _pd]),
}


class EdgError(RuntimeError):
    """A negative EDG_* status from the engine, with the engine's message."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"libedgpu.so not built at {path}; run `python ed_lattice_b200/build.py`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def check(status: int, where: str) -> None:
    if status != EDG_OK:
        msg = lib().edg_last_error()
        raise EdgError(status, where, msg.decode() if msg else "")
