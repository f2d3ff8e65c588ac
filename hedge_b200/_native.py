"""ctypes binding of libhedge_b200.so (the C ABI in include/hedge_b200.h).

The library is built in-tree (hedge_b200/build.py).  There is no CPU
fallback: if the library is missing or a call fails, an exception is raised.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhedge_b200.so")

HB_OK, HB_ERR_INVALID_ARGUMENT, HB_ERR_UNSUPPORTED, HB_ERR_CUDA, HB_ERR_DEVICE_FLAG = range(5)
PREC_FP64, PREC_FP32, PREC_BF16X3, PREC_FP16X3, PREC_FP32_SIMT = 0, 1, 2, 3, 4


class HedgeB200Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("hedge_b200 error %d: %s" % (status, msg))
        self.status = status


class ValueErrorStatus(HedgeB200Error, ValueError):
    pass


class hb_discr_desc(C.Structure):
    _fields_ = [("dim", C.c_int32), ("order", C.c_int32), ("np", C.c_int32),
                ("nfp", C.c_int32), ("nfaces", C.c_int32), ("nperm", C.c_int32),
                ("num_elements", C.c_int64),
                ("dmats", C.c_void_p), ("lift", C.c_void_p), ("geometry", C.c_void_p),
                ("fmask", C.c_void_p), ("shuffle", C.c_void_p),
                ("device", C.c_int32), ("unit_nodes", C.c_void_p),
                ("mass", C.c_void_p), ("abs_jacobian", C.c_void_p)]


class hb_batch_member(C.Structure):
    _fields_ = [("op", C.c_void_p), ("q0", C.c_void_p), ("q1", C.c_void_p),
                ("res", C.c_void_p), ("dt", C.c_double), ("tile_elems", C.c_int32)]


class hb_quad_desc(C.Structure):
    _fields_ = [("nq", C.c_int32), ("nqf", C.c_int32),
                ("vol_interp", C.c_void_p), ("vol_project", C.c_void_p),
                ("face_interp", C.c_void_p), ("face_lift", C.c_void_p)]


class hb_op_desc(C.Structure):
    _fields_ = [("model", C.c_int32), ("num_fields", C.c_int32),
                ("precision", C.c_int32), ("flux_type", C.c_int32),
                ("bdry_flux_type", C.c_int32),
                ("v", C.c_double * 3), ("c", C.c_double), ("eps", C.c_double),
                ("mu", C.c_double), ("alpha", C.c_double), ("bdry_alpha", C.c_double),
                ("time_sign", C.c_double),
                ("conn", C.c_void_p), ("num_given_bdry_nodes", C.c_int64),
                ("num_halo_faces", C.c_int64),
                ("quadrature", C.POINTER(hb_quad_desc))]


EXPORTED = [
    "hb_discr_create", "hb_discr_destroy", "hb_op_create", "hb_op_destroy",
    "hb_rhs", "hb_lsrk_stage", "hb_rhs_elements", "hb_lsrk_stage_elements", "hb_lincomb",
    "hb_gather_map", "hb_op_check",
    "hb_op_launch_info", "hb_norm", "hb_norm_noalloc", "hb_rhs_adjoint_work_size",
    "hb_rhs_adjoint", "hb_batch_create", "hb_batch_destroy", "hb_batch_stage",
    "hb_batch_info", "hb_batch_check", "hb_op_set_halo", "hb_pack",
    "hb_op_wait_selftest", "hb_last_error_string",
]

_lib = None
_lock = threading.Lock()


def load(path=LIB_PATH):
    """Load (once) and return the ctypes library with typed signatures."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                "libhedge_b200.so not found at %s; build it with "
                "`python -m hedge_b200.build`" % path)
        lib = C.CDLL(path)
        vp, i32, i64, d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        sig = {
            "hb_discr_create": [C.POINTER(hb_discr_desc), C.POINTER(vp)],
            "hb_discr_destroy": [vp],
            "hb_op_create": [vp, C.POINTER(hb_op_desc), C.POINTER(vp)],
            "hb_op_destroy": [vp],
            "hb_rhs": [vp, vp, vp, vp, vp, vp, vp],
            "hb_lsrk_stage": [vp, d, d, d, vp, vp, vp, vp, vp, vp, vp],
            "hb_rhs_elements": [vp, i64, i64, vp, vp, vp, vp, vp, vp],
            "hb_lsrk_stage_elements": [vp, i64, i64, d, d, d, vp, vp, vp, vp, vp, vp, vp],
            "hb_lincomb": [i64, i32, d, vp, d, vp, vp, vp],
            "hb_gather_map": [vp, vp, vp, vp],
            "hb_op_check": [vp, vp],
            "hb_op_launch_info": [vp, vp, i32],
            "hb_norm": [vp, i32, i32, vp, vp, vp],
            "hb_norm_noalloc": [i64, i32, i32, i32, vp, vp, vp, vp, vp],
            "hb_rhs_adjoint_work_size": [vp, vp],
            "hb_rhs_adjoint": [vp, vp, vp, vp, vp, vp, vp, vp],
            "hb_batch_create": [vp, i32, vp],
            "hb_batch_destroy": [vp],
            "hb_batch_stage": [vp, d, d, i32, vp],
            "hb_batch_info": [vp, vp, i32],
            "hb_batch_check": [vp, vp],
            "hb_op_set_halo": [vp, vp, vp],
            "hb_pack": [i64, i32, i32, i64, vp, vp, vp, vp],
            "hb_op_wait_selftest": [vp, i64, vp],
        }
        for name, args in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = C.c_int
        lib.hb_last_error_string.argtypes = []
        lib.hb_last_error_string.restype = C.c_char_p
        _lib = lib
        return lib


def check(status):
    if status != HB_OK:
        msg = load().hb_last_error_string().decode(errors="replace")
        cls = ValueErrorStatus if status == HB_ERR_INVALID_ARGUMENT else HedgeB200Error
        raise cls(status, msg)
    return status
