"""ctypes binding of libprandtl_b200.so (the C ABI in include/prandtl_b200.h).

The library is built in-tree (``python -m prandtl_b200.build``).  There is no
CPU fallback: if the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libprandtl_b200.so")

PRANDTL_OK, PRANDTL_EINVAL, PRANDTL_ENOMEM, PRANDTL_ENONFINITE = 0, 1, 2, 3
PRANDTL_ETIMEDOUT, PRANDTL_ECUDA, PRANDTL_EUNSUPPORTED, PRANDTL_ETOOLARGE = 4, 5, 6, 7
PTR_HOST, PTR_DEVICE = 0, 1
KERNEL_RHS, KERNEL_LIFT = 0, 1
RK3SSP, LSRK45 = 0, 1

STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ENONFINITE", 4: "ETIMEDOUT",
                5: "ECUDA", 6: "EUNSUPPORTED", 7: "ETOOLARGE"}

# Every symbol include/prandtl_b200.h declares.
EXPORTS = ["prandtl_config_default", "prandtl_create", "prandtl_destroy", "prandtl_rhs",
           "prandtl_step", "prandtl_get_alpha", "prandtl_cfl_dt", "prandtl_set_stream",
           "prandtl_synchronize", "prandtl_kernel_launches", "prandtl_profile",
           "prandtl_profile_read", "prandtl_profile_reset", "prandtl_device_bytes",
           "prandtl_last_error", "prandtl_version", "prandtl_rhs_noalloc"]


class MeshDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("order", C.c_int), ("num_elements", C.c_int),
                ("num_faces", C.c_int), ("elem_adj", C.POINTER(C.c_double)),
                ("elem_detj", C.POINTER(C.c_double)), ("face_elems", C.POINTER(C.c_int)),
                ("face_nor", C.POINTER(C.c_double))]


class Config(C.Structure):
    _fields_ = [("gamma", C.c_double), ("Pr", C.c_double), ("mu", C.c_double),
                ("R_gas", C.c_double), ("alpha_max", C.c_double), ("alpha_min", C.c_double),
                ("parabolic", C.c_int), ("blending", C.c_int), ("sutherland", C.c_int),
                ("quirks", C.c_int), ("surface_dissipation", C.c_int), ("precision", C.c_int),
                ("timeout_s", C.c_double)]


class PrandtlError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"prandtl {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_LIB = None


def load():
    """Load (never build) the in-tree library and declare its signatures."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise PrandtlError(PRANDTL_ECUDA, f"{LIB_PATH} is missing; run python -m prandtl_b200.build")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
    L.prandtl_config_default.argtypes = [C.POINTER(Config)]
    L.prandtl_config_default.restype = None
    L.prandtl_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Config), C.POINTER(vp)]
    L.prandtl_create.restype = ip
    L.prandtl_destroy.argtypes = [vp]
    L.prandtl_destroy.restype = ip
    L.prandtl_rhs.argtypes = [vp, vp, vp, C.c_double, dp, ip]
    L.prandtl_rhs.restype = ip
    L.prandtl_step.argtypes = [vp, vp, C.c_double, C.c_double, ip, ip, ip]
    L.prandtl_step.restype = ip
    L.prandtl_get_alpha.argtypes = [vp, vp, ip]
    L.prandtl_get_alpha.restype = ip
    L.prandtl_cfl_dt.argtypes = [C.c_double, C.c_double, C.c_double, ip]
    L.prandtl_cfl_dt.restype = C.c_double
    L.prandtl_set_stream.argtypes = [vp, vp]
    L.prandtl_set_stream.restype = ip
    L.prandtl_synchronize.argtypes = [vp]
    L.prandtl_synchronize.restype = ip
    L.prandtl_kernel_launches.argtypes = [vp]
    L.prandtl_kernel_launches.restype = C.c_longlong
    L.prandtl_profile.argtypes = [vp, ip]
    L.prandtl_profile.restype = ip
    L.prandtl_profile_read.argtypes = [vp, ip, dp, C.POINTER(C.c_longlong)]
    L.prandtl_profile_read.restype = ip
    L.prandtl_profile_reset.argtypes = [vp]
    L.prandtl_profile_reset.restype = ip
    L.prandtl_device_bytes.argtypes = [vp]
    L.prandtl_device_bytes.restype = C.c_size_t
    L.prandtl_last_error.argtypes = [vp]
    L.prandtl_last_error.restype = C.c_char_p
    L.prandtl_rhs_noalloc.argtypes = [C.POINTER(MeshDesc), C.POINTER(Config), vp, vp, vp]
    L.prandtl_rhs_noalloc.restype = ip
    L.prandtl_version.argtypes = []
    L.prandtl_version.restype = C.c_char_p
    _LIB = L
    return L


def check(status, handle=None):
    if status != PRANDTL_OK:
        msg = load().prandtl_last_error(handle).decode(errors="replace")
        raise PrandtlError(status, msg)
