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
           "prandtl_last_error", "prandtl_version", "prandtl_rhs_noalloc", "prandtl_recover_state",
           "prandtl_budgets", "prandtl_batch_budgets",
           "prandtl_batch_config_default", "prandtl_batch_create", "prandtl_batch_destroy",
           "prandtl_batch_footprint", "prandtl_batch_add", "prandtl_batch_add_many", "prandtl_batch_advance",
           "prandtl_batch_sync", "prandtl_batch_finished", "prandtl_batch_query",
           "prandtl_batch_read", "prandtl_batch_read_many", "prandtl_batch_remove", "prandtl_batch_tune", "prandtl_batch_tune_in_steps",
           "prandtl_batch_class_info", "prandtl_batch_stream", "prandtl_batch_device_bytes",
           "prandtl_batch_arena_bytes", "prandtl_batch_time",
           "prandtl_batch_kernel_launches", "prandtl_batch_last_error",
           "prandtl_serve_create", "prandtl_serve_submit", "prandtl_serve_poll",
           "prandtl_serve_wait", "prandtl_serve_stats_get", "prandtl_serve_destroy",
           "prandtl_serve_last_error",
           "prandtl_mesh_read", "prandtl_mesh_describe", "prandtl_mesh_face_attributes",
           "prandtl_mesh_element_attributes", "prandtl_mesh_set_boundary_conditions",
           "prandtl_mesh_attribute", "prandtl_mesh_node_coords", "prandtl_mesh_destroy",
           "prandtl_mesh_last_error", "prandtl_checkpoint_save", "prandtl_checkpoint_load",
           "prandtl_paraview_save", "prandtl_io_last_error"]


class MeshDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("order", C.c_int), ("num_elements", C.c_int),
                ("num_faces", C.c_int), ("elem_adj", C.POINTER(C.c_double)),
                ("elem_detj", C.POINTER(C.c_double)), ("face_elems", C.POINTER(C.c_int)),
                ("face_nor", C.POINTER(C.c_double)), ("node_adj", C.POINTER(C.c_double)),
                ("node_detj", C.POINTER(C.c_double)), ("face_node_nor", C.POINTER(C.c_double))]


class BC(C.Structure):
    _fields_ = [("type", C.c_int), ("state", C.c_double * 5), ("p", C.c_double), ("pt", C.c_double),
                ("Tt", C.c_double), ("cp", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
                ("wall_vel", C.c_double * 3), ("heat_flux", C.c_double), ("wall_T", C.c_double)]


BC_TYPES = {"state": 0, "outflow": 1, "slip_wall": 2, "symmetry": 3, "pressure_outflow": 4,
            "riemann": 5, "inflow_rv": 6, "inflow_pttt": 7, "noslip_adiabatic": 8, "noslip_isothermal": 9,
            "axis": 10}


class Config(C.Structure):
    _fields_ = [("gamma", C.c_double), ("Pr", C.c_double), ("mu", C.c_double),
                ("R_gas", C.c_double), ("alpha_max", C.c_double), ("alpha_min", C.c_double),
                ("parabolic", C.c_int), ("blending", C.c_int), ("sutherland", C.c_int),
                ("quirks", C.c_int), ("surface_dissipation", C.c_int), ("precision", C.c_int),
                ("timeout_s", C.c_double), ("num_bcs", C.c_int), ("bcs", C.POINTER(BC)),
                ("axisymmetric", C.c_int), ("node_coords", C.POINTER(C.c_double)),
                ("axis_rho_floor", C.c_double)]


class BatchConfig(C.Structure):
    _fields_ = [("precision", C.c_int), ("scheme", C.c_int), ("arena_bytes", C.c_size_t),
                ("max_solves", C.c_int), ("steps_per_graph", C.c_int), ("use_graph", C.c_int),
                ("timeout_s", C.c_double)]


class SolveDesc(C.Structure):
    _fields_ = [("dt", C.c_double), ("cfl", C.c_double), ("hmin", C.c_double), ("nsteps", C.c_int),
                ("t_final", C.c_double)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("rejected", C.c_longlong),
                ("steps", C.c_longlong), ("dof_updates", C.c_double), ("busy_s", C.c_double),
                ("resident", C.c_int)]


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
    L.prandtl_recover_state.argtypes = [vp, vp, vp, ip]
    L.prandtl_recover_state.restype = ip
    L.prandtl_budgets.argtypes = [vp, vp, vp, vp, ip]
    L.prandtl_budgets.restype = ip
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
    # batches
    bcp, sdp, mdp, cfp = C.POINTER(BatchConfig), C.POINTER(SolveDesc), C.POINTER(MeshDesc), C.POINTER(Config)
    ipp = C.POINTER(C.c_int)
    sig = {
        "prandtl_batch_config_default": (None, [bcp]),
        "prandtl_batch_create": (ip, [bcp, C.POINTER(vp)]),
        "prandtl_batch_destroy": (ip, [vp]),
        "prandtl_batch_footprint": (ip, [vp, mdp, cfp, C.POINTER(C.c_size_t)]),
        "prandtl_batch_add": (ip, [vp, mdp, cfp, vp, ip, sdp, ipp]),
        "prandtl_batch_add_many": (ip, [vp, ip, vp, vp, vp, ip, vp, vp]),
        "prandtl_batch_advance": (ip, [vp, ip]),
        "prandtl_batch_sync": (ip, [vp]),
        "prandtl_batch_finished": (ip, [vp, ipp, ip, ipp]),
        "prandtl_batch_query": (ip, [vp, ip, ipp, ipp, dp, dp]),
        "prandtl_batch_read": (ip, [vp, ip, vp, ip]),
        "prandtl_batch_read_many": (ip, [vp, ip, vp, vp, ip]),
        "prandtl_batch_time": (ip, [vp, ip, dp]),
        "prandtl_batch_budgets": (ip, [vp, ip, vp]),
        "prandtl_batch_remove": (ip, [vp, ip]),
        "prandtl_batch_tune": (ip, [vp, ip]),
        "prandtl_batch_tune_in_steps": (ip, [vp]),
        "prandtl_batch_class_info": (ip, [vp, ip, ip, ip, ipp, ipp, dp, dp]),
        "prandtl_batch_stream": (vp, [vp]),
        "prandtl_batch_device_bytes": (C.c_size_t, [vp]),
        "prandtl_batch_arena_bytes": (C.c_size_t, [vp]),
        "prandtl_batch_kernel_launches": (C.c_longlong, [vp]),
        "prandtl_batch_last_error": (C.c_char_p, [vp]),
        "prandtl_serve_create": (ip, [bcp, ip, C.POINTER(vp)]),
        "prandtl_serve_submit": (ip, [vp, mdp, cfp, vp, sdp, vp, C.POINTER(C.c_longlong)]),
        "prandtl_serve_poll": (ip, [vp, C.c_longlong, ipp, dp]),
        "prandtl_serve_wait": (ip, [vp, C.c_longlong, C.c_double, dp]),
        "prandtl_serve_stats_get": (ip, [vp, C.POINTER(ServeStats)]),
        "prandtl_serve_destroy": (ip, [vp]),
        "prandtl_serve_last_error": (C.c_char_p, [vp]),
        "prandtl_mesh_read": (ip, [C.c_char_p, ip, ip, ip, C.POINTER(vp)]),
        "prandtl_mesh_describe": (ip, [vp, mdp, dp]),
        "prandtl_mesh_face_attributes": (ip, [vp, ipp]),
        "prandtl_mesh_element_attributes": (ip, [vp, ipp]),
        "prandtl_mesh_set_boundary_conditions": (ip, [vp, ipp, ip]),
        "prandtl_mesh_attribute": (ip, [vp, ip, C.c_char_p]),
        "prandtl_mesh_node_coords": (ip, [vp, dp]),
        "prandtl_mesh_destroy": (None, [vp]),
        "prandtl_mesh_last_error": (C.c_char_p, []),
        "prandtl_checkpoint_save": (ip, [C.c_char_p, ip, C.c_double, ip, ip, ip, C.c_longlong, dp]),
        "prandtl_checkpoint_load": (ip, [C.c_char_p, ip, ip, ip, ip, C.c_longlong, dp, dp]),
        "prandtl_paraview_save": (ip, [C.c_char_p, C.c_char_p, ip, C.c_double, ip, ip, ip, dp, dp, dp,
                                       C.c_double, ip]),
        "prandtl_io_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def check(status, handle=None, last_error=None):
    """Raise PrandtlError for a non-OK status with the object's last error text
    (`last_error` names the getter: prandtl_last_error by default)."""
    if status != PRANDTL_OK:
        getter = getattr(load(), last_error or "prandtl_last_error")
        msg = getter(handle).decode(errors="replace")
        raise PrandtlError(status, msg)
