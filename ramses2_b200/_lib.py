"""Loader of librh_b200.so, the in-tree sm_100a CUDA library.

There is no CPU fallback: if the library is missing or cannot be loaded, every
entry point of this package raises.
"""
import ctypes as C
import os

from ._abi import STATUS, BatchIC, BatchProblem, FlagParams, HydroParams, MeshDesc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librh_b200.so")

_lib = None

# name -> (restype, argtypes); mirrors include/ramses_hydro.h and the
# extension entry points declared in include/ramses_hydro_ext.h
_P = C.POINTER
_d = C.c_double
_i = C.c_int
SIGNATURES = {
    "rh_init": (_i, [_i]),
    "rh_finalize": (_i, []),
    "rh_last_error": (C.c_char_p, []),
    "rh_sync": (_i, []),
    "rh_set_precision": (_i, [_i]),
    "rh_set_mesh": (_i, [_P(MeshDesc), _P(_d), _i, _i]),
    "rh_set_grid_device": (_i, [_P(_d), _i, _i, _i]),
    "rh_transfer_grid_host": (_i, [_P(_d), _i, _i, _i]),
    "rh_set_unew": (_i, [_i, _i]),
    "rh_set_uold": (_i, [_i, _i]),
    "rh_cmpdt": (_i, [_i, _i, _d, _d, _d, _d, _d, _P(_d), _P(_d), _P(_d), _P(_d), _P(_d), _P(_d)]),
    "rh_godunov": (_i, [_i, _i, _i, _i, _i, _i, _d, _d, _d, _d, _d, _d, _i, _i, _P(_d)]),
    "rh_set_interpolation": (_i, [_i, _i]),
    "rh_upload": (_i, [_i, _i, _i, _d, _d, _d]),
    "rh_hydro_flag": (_i, [_i, _P(FlagParams), _d, _d, _P(C.c_int32), _P(C.c_longlong)]),
    # extensions (include/ramses_hydro_ext.h)
    "rh_set_tile": (_i, [_i, _i, _i, _i]),
    "rh_set_amr_tile": (_i, [_i, _i, _i, _i]),
    "rh_get_tile": (_i, [_P(_i), _P(_i), _P(_i), _P(_i)]),
    "rh_list_tiles": (_i, [_i, _P(_i), _P(_i), _P(_i), _i]),
    "rh_level_info": (_i, [_i, _P(_i), _P(C.c_longlong)]),
    "rh_level_table": (_i, [_i, _P(_i), _P(C.c_longlong), _P(_i), C.c_longlong]),
    "rh_level_ghosts": (_i, [_i, _P(_i), _P(C.c_ubyte), _P(_i), C.c_longlong]),
    "rh_set_table_builder": (_i, [_i]),
    "rh_set_deterministic": (_i, [_i]),
    "rh_coarse_step": (_i, [_P(HydroParams), _P(_d), _P(_d)]),
    "rh_coarse_step_host": (_i, [_P(HydroParams), C.c_void_p, C.c_void_p, _P(_d), _P(_d)]),
    "rh_state_ptrs": (_i, [_P(C.c_void_p), _P(C.c_void_p), _P(C.c_void_p), _P(C.c_void_p)]),
    "rh_bench_godunov": (_i, [_i, _i, _d, _d, _d, _d, _d, _d, _i, _i, _P(C.c_float)]),
    "rh_timer_start": (_i, []),
    "rh_timer_stop": (_i, [_P(C.c_float)]),
    "rh_selftest_wait": (_i, [C.c_longlong]),
    "rh_selftest_vmath": (_i, [C.c_void_p, C.c_longlong, C.c_void_p]),
    "rh_check_state": (_i, [_i, _i, _P(_i), _P(_i), _P(_i)]),
    "rh_set_state_check": (_i, [_i]),
    # restart / snapshot files (include/ramses_hydro_io.h)
    "rh_file_size": (_i, [_i, _P(C.c_longlong)]),
    "rh_file_image": (_i, [_i, _d, C.c_void_p, C.c_longlong, _P(C.c_longlong)]),
    "rh_file_image_device": (_i, [_i, _d, _P(C.c_void_p), _P(C.c_longlong)]),
    "rh_restore_hydro": (_i, [C.c_void_p, C.c_longlong]),
    "rh_batch_file_image": (_i, [_i, _i, C.c_void_p, C.c_longlong, _P(C.c_longlong)]),
    # batch (include/ramses_hydro_batch.h)
    "rh_batch_init": (_i, [_i, _i, _i, C.c_longlong]),
    "rh_batch_free": (_i, []),
    "rh_batch_footprint": (C.c_longlong, [_P(BatchProblem)]),
    "rh_batch_add": (_i, [_P(BatchProblem), _P(BatchIC), _P(_i)]),
    "rh_batch_remove": (_i, [_i]),
    "rh_batch_step": (_i, [_i]),
    "rh_batch_status": (_i, [_i, _P(_d), _P(_i), _P(_i), _P(_d), _P(_d)]),
    "rh_batch_poll": (_i, [_P(_i), _P(_i), _P(_d)]),
    "rh_batch_capacity": (_i, []),
    "rh_batch_fetch": (_i, [_i, _P(_d)]),
    "rh_batch_set_tile": (_i, [_i, _i, _i, _i]),
    "rh_batch_list_tiles": (_i, [_i, _P(_i), _P(_i), _P(_i), _i]),
    "rh_batch_bench": (_i, [_i, _P(C.c_float)]),
    "rh_batch_cells": (C.c_longlong, []),
    "rh_batch_set_plane_path": (_i, [_i]),
    "rh_batch_set_state_check": (_i, [_i]),
    "rh_batch_check_mask": (_i, [_i, _P(_i)]),
}


class RHError(RuntimeError):
    pass


def lib():
    """Load (and type) librh_b200.so; raise if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RHError("librh_b200.so is not built: run `python -m ramses2_b200.build` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc, what=""):
    if rc != 0:
        msg = lib().rh_last_error().decode()
        raise RHError("%s failed: %s (%s)" % (what or "rh call", STATUS.get(rc, rc), msg))
    return rc
