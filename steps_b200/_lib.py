"""ctypes binding of the C ABI in include/steps_b200.h (libsteps_b200.so).

The library is built in-tree by ``steps_b200.build``.  There is no fallback: if the
shared library is missing, loading fails with the build command.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# STEPS_B200_LIB may point at another build of the same sources (e.g. a tuning variant).
LIB_PATH = os.environ.get("STEPS_B200_LIB") or os.path.join(_HERE, "libsteps_b200.so")


class StepsError(RuntimeError):
    """Base of the errors raised through the C ABI (reference: steps::Err)."""


class ArgErr(StepsError):
    pass


class ProgErr(StepsError):
    pass


class NotImplErr(StepsError):
    pass


class CudaError(StepsError):
    pass


class DeviceError(StepsError):
    pass


_ERRS = {1: ArgErr, 2: ProgErr, 3: NotImplErr, 4: CudaError, 5: DeviceError}

_i32, _u32, _u64, _f64 = C.c_int32, C.c_uint32, C.c_uint64, C.c_double
_P = C.c_void_p
_pi32, _pu32, _pf64, _pu64 = (C.POINTER(C.c_int32), C.POINTER(C.c_uint32),
                              C.POINTER(C.c_double), C.POINTER(C.c_uint64))

# name -> argument types (all return int status)
PROTOTYPES = {
    "sg_create": [C.POINTER(_P), _u64, C.c_int],
    "sg_destroy": [_P],
    "sg_set_nspecs": [_P, _i32],
    "sg_set_mesh": [_P, _i32, _pf64, _pi32, _pf64, _pf64, _pi32, _i32],
    "sg_set_diff_boundaries": [_P, _i32, _pi32, _pi32],
    "sg_set_diff_boundary_active": [_P, _i32, _i32, _i32],
    "sg_get_diff_boundary_active": [_P, _i32, _i32, _pi32],
    "sg_set_diff_boundary_dcst": [_P, _i32, _i32, _f64, _i32],
    "sg_add_reac": [_P, _i32, _pu32, _pi32, _f64, _pi32],
    "sg_add_diff": [_P, _i32, _i32, _f64, _pi32],
    "sg_set_realizations": [_P, _i32, _pi32],
    "sg_setup": [_P],
    "sg_reset": [_P],
    "sg_run": [_P, _f64],
    "sg_advance": [_P, _f64],
    "sg_get_time": [_P, _pf64],
    "sg_get_update_period": [_P, _i32, _pf64],
    "sg_get_nsteps": [_P, _pu64],
    "sg_get_niteration": [_P, _pu64],
    "sg_get_reac_extent": [_P, _i32, _pu64],
    "sg_get_diff_extent": [_P, _pu64],
    "sg_set_diff_apply_threshold": [_P, _i32],
    "sg_get_tet_count": [_P, _i32, _i32, _pf64],
    "sg_set_tet_count": [_P, _i32, _i32, _f64],
    "sg_get_comp_count": [_P, _i32, _i32, _i32, _pf64],
    "sg_set_comp_count": [_P, _i32, _i32, _i32, _f64],
    "sg_get_spec_counts": [_P, _i32, _pu32],
    "sg_get_batch_tet_counts": [_P, _i32, _pi32, _i32, _pf64],
    "sg_set_spec_counts": [_P, _i32, _pu32],
    "sg_get_all_counts": [_P, _pu32],
    "sg_set_all_counts": [_P, _pu32],
    "sg_set_tet_clamped": [_P, _i32, _i32, _i32],
    "sg_set_reac_k": [_P, _i32, _i32, _f64],
    "sg_get_reac_k": [_P, _i32, _i32, _pf64],
    "sg_set_diff_d": [_P, _i32, _i32, _i32, _f64],
    "sg_checkpoint": [_P, C.c_char_p],
    "sg_restore": [_P, C.c_char_p],
    "sg_set_launch": [_P, _i32, _i32],
    "sg_get_launch": [_P, _pi32, _pi32],
    "sg_set_autotune": [_P, _i32],
    "sg_get_carveout": [_P, _pi32],
    "sg_set_split": [_P, _i32],
    "sg_get_split": [_P, _pi32],
    "sg_set_persistent": [_P, _i32, _i32],
    "sg_get_persistent": [_P, _pi32, _pi32],
    "sg_set_window_wait_limit": [_P, C.c_uint32],
    "sg_get_autotune_ms": [_P, C.POINTER(C.c_float), _i32, _pi32],
    "sg_set_conservation_check": [_P, _i32],
    "sg_set_graphs": [_P, _i32],
    "sg_get_status": [_P, _pu32],
    "sg_set_surface": [_P, _i32, _i32, _pi32, _pi32, _pf64, _i32],
    "sg_add_sreac": [_P, _i32, _pu32, _pu32, _pi32, _pi32, _f64, _pi32],
    "sg_set_tri_outer": [_P, _pi32],
    "sg_set_sreac_outer": [_P, _i32, _pu32, _pi32],
    "sg_add_vdep_sreac": [_P, _i32, _pu32, _pu32, _pi32, _pi32, _f64, _f64, _i32, _pf64, _pi32],
    "sg_add_ghk": [_P, _i32, _i32, _i32, _i32, _f64, _f64, _f64, _i32, _pi32],
    "sg_set_temp": [_P, _f64],
    "sg_get_temp": [_P, _pf64],
    "sg_get_tri_ghk_i": [_P, _i32, _pf64],
    "sg_set_tri_neighbours": [_P, _pi32, _pi32, _pf64, _pf64],
    "sg_add_sdiff": [_P, _i32, _i32, _f64, _pi32],
    "sg_add_ohmic": [_P, _i32, _i32, _f64, _f64, _pi32],
    "sg_get_tri_count": [_P, _i32, _i32, _pf64],
    "sg_set_tri_count": [_P, _i32, _i32, _f64],
    "sg_get_patch_count": [_P, _i32, _i32, _i32, _pf64],
    "sg_set_patch_count": [_P, _i32, _i32, _i32, _f64],
    "sg_get_tri_ohmic_i": [_P, _i32, _pf64],
    "sg_set_efield_mesh": [_P, _i32, _pf64, _pi32, _i32, _pi32, _i32],
    "sg_set_efield_dt": [_P, _f64],
    "sg_get_efield_dt": [_P, _pf64],
    "sg_set_efield_tolerance": [_P, _f64, _f64, _i32],
    "sg_set_memb_potential": [_P, _f64],
    "sg_set_memb_capac": [_P, _f64],
    "sg_set_memb_vol_res": [_P, _f64],
    "sg_set_memb_res": [_P, _f64, _f64],
    "sg_get_vert_v": [_P, _i32, _pf64],
    "sg_set_vert_v": [_P, _i32, _f64],
    "sg_get_tri_v": [_P, _i32, _pf64],
    "sg_set_vert_v_clamped": [_P, _i32, _i32],
    "sg_set_vert_iclamp": [_P, _i32, _f64],
    "sg_get_efield_stats": [_P, _pu64, _pu64, _pf64, _pf64],
    "sg_set_efield_check": [_P, _i32, _f64],
    "sg_set_efield_persistent": [_P, _i32],
    "sg_set_efield_barrier_limit": [_P, _u32],
    "sg_set_efield_reliable_updates": [_P, _i32, _f64],
    "sg_get_efield_check": [_P, _pu64, _pf64, _pf64],
    "sg_get_stream": [_P, C.POINTER(_P)],
    "sg_set_profiling": [_P, _i32],
    "sg_get_profile": [_P, _pf64, _pu64, _pu64],
}

_lib = None


def load():
    """Load libsteps_b200.so and declare every prototype; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m steps_b200.build` "
            "(nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(LIB_PATH)
    for name, args in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    lib.sg_last_error.argtypes = []
    lib.sg_last_error.restype = C.c_char_p
    lib.sg_version.argtypes = []
    lib.sg_version.restype = C.c_int
    _lib = lib
    return lib


def check(status):
    if status != 0:
        msg = _lib.sg_last_error().decode("utf-8", "replace")
        raise _ERRS.get(status, StepsError)(msg)


def ptr(arr, ctype):
    """Pointer to a contiguous numpy array's data as the given ctypes type."""
    return arr.ctypes.data_as(C.POINTER(ctype))
