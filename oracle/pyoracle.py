"""ctypes binding of the CPU oracle (liboracle.so).

Test infrastructure: imported only by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OracleMesh(C.Structure):
    _fields_ = [("dim", C.c_int), ("order", C.c_int), ("num_elements", C.c_int),
                ("num_faces", C.c_int), ("elem_adj", C.POINTER(C.c_double)),
                ("elem_detj", C.POINTER(C.c_double)), ("face_elems", C.POINTER(C.c_int)),
                ("face_nor", C.POINTER(C.c_double)), ("node_adj", C.POINTER(C.c_double)),
                ("node_detj", C.POINTER(C.c_double)), ("face_node_nor", C.POINTER(C.c_double))]


def _node_geometry(mesh, dtype):
    """Per-node adjugates / determinants and per-face-node normals of a mesh with
    non-affine elements (None for affine meshes)."""
    if getattr(mesh, "node_adj", None) is None:
        return None
    return tuple(np.ascontiguousarray(a, dtype=dtype) for a in (mesh.node_adj, mesh.node_detj, mesh.face_node_nor))


class OracleBC(C.Structure):
    _fields_ = [("type", C.c_int), ("state", C.c_double * 5), ("p", C.c_double), ("pt", C.c_double),
                ("Tt", C.c_double), ("cp", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
                ("wall_vel", C.c_double * 3), ("heat_flux", C.c_double), ("wall_T", C.c_double)]


# boundary-condition types (prandtl_oracle.h ORACLE_BC_*)
BC_TYPES = {"state": 0, "outflow": 1, "slip_wall": 2, "symmetry": 3, "pressure_outflow": 4,
            "riemann": 5, "inflow_rv": 6, "inflow_pttt": 7, "noslip_adiabatic": 8, "noslip_isothermal": 9,
            "axis": 10}


class OracleConfig(C.Structure):
    _fields_ = [("gamma", C.c_double), ("Pr", C.c_double), ("mu", C.c_double),
                ("R_gas", C.c_double), ("alpha_max", C.c_double), ("alpha_min", C.c_double),
                ("parabolic", C.c_int), ("blending", C.c_int), ("sutherland", C.c_int),
                ("quirks", C.c_int), ("surface_dissipation", C.c_int),
                ("num_bcs", C.c_int), ("bcs", C.POINTER(OracleBC)),
                ("axisymmetric", C.c_int), ("node_coords", C.POINTER(C.c_double)),
                ("axis_rho_floor", C.c_double)]


def make_bcs(bcs):
    """ctypes array of boundary conditions from [(type name, state or None, p or None), ...];
    for inflow_pttt and the no-slip walls the second item is a dict of named fields."""
    if not bcs:
        return None
    arr = (OracleBC * len(bcs))()
    for k, b in enumerate(bcs):
        kind, state, p = (tuple(b) + (None, None))[:3]
        arr[k].type = BC_TYPES[kind]
        if isinstance(state, dict):   # inflow_pttt, noslip_*: named fields
            for name, v in state.items():
                if name == "wall_vel":
                    for d, x in enumerate(v):
                        arr[k].wall_vel[d] = float(x)
                else:
                    setattr(arr[k], name, float(v))
        else:
            for f, v in enumerate(state if state is not None else []):
                arr[k].state[f] = float(v)
        arr[k].p = float(p) if p is not None else 0.0
    return arr


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        L.oracle_rhs.argtypes = [C.POINTER(OracleMesh), C.POINTER(OracleConfig), dp, dp, dp, dp, dp, C.c_int]
        L.oracle_rhs.restype = C.c_int
        L.oracle_step.argtypes = [C.POINTER(OracleMesh), C.POINTER(OracleConfig), dp, C.c_double,
                                  C.c_double, C.c_int, C.c_int, C.c_int]
        L.oracle_step.restype = C.c_int
        L.oracle_recover_weighted.argtypes = [C.POINTER(OracleMesh), C.POINTER(OracleConfig), dp, dp]
        L.oracle_recover_weighted.restype = C.c_int
        L.oracle_gl.argtypes = [C.c_int, dp, dp, dp]
        L.oracle_log_mean.argtypes = [C.c_double, C.c_double]
        L.oracle_log_mean.restype = C.c_double
        L.oracle_volume_flux.argtypes = [C.c_int, C.c_double, dp, dp, dp, dp, dp]
        L.oracle_volume_flux.restype = C.c_double
        L.oracle_face_flux.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, dp, dp, dp, dp]
        L.oracle_face_flux.restype = C.c_double
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """Holds one mesh + physics configuration for repeated oracle calls."""

    def __init__(self, mesh, gamma=1.4, Pr=0.72, mu=0.02, R_gas=287.05, alpha_max=0.5,
                 alpha_min=0.001, parabolic=0, blending=0, sutherland=0, quirks=0,
                 surface_dissipation=1, nthreads=None, bcs=None, axisymmetric=0,
                 axis_rho_floor=0.0):
        self.mesh = mesh
        self._adj = np.ascontiguousarray(mesh.elem_adj, dtype=np.float64)
        self._detj = np.ascontiguousarray(mesh.elem_detj, dtype=np.float64)
        self._faces = np.ascontiguousarray(mesh.face_elems, dtype=np.int32)
        self._nor = np.ascontiguousarray(mesh.face_nor, dtype=np.float64)
        self._ngeo = _node_geometry(mesh, np.float64)
        ng = [_p(a) for a in self._ngeo] if self._ngeo else [None, None, None]
        self.m = OracleMesh(mesh.dim, mesh.order, mesh.num_elements, mesh.num_faces,
                            _p(self._adj), _p(self._detj),
                            self._faces.ctypes.data_as(C.POINTER(C.c_int)), _p(self._nor), *ng)
        self._bcs = make_bcs(bcs)
        self._xy = np.ascontiguousarray(mesh.coords, dtype=np.float64)
        self.c = OracleConfig(gamma, Pr, mu, R_gas, alpha_max, alpha_min, parabolic, blending,
                              sutherland, quirks, surface_dissipation, len(bcs) if bcs else 0,
                              self._bcs, int(axisymmetric), _p(self._xy), float(axis_rho_floor))
        self.nthreads = nthreads or os.cpu_count() or 1

    @property
    def size(self):
        return self.mesh.num_fields * self.mesh.ndof

    def rhs(self, u, want_alpha=False, want_grad=False):
        u = np.ascontiguousarray(u, dtype=np.float64)
        dudt = np.empty_like(u)
        alpha = np.empty(self.mesh.num_elements) if want_alpha else None
        lam = np.zeros(1)
        grad = np.empty(self.mesh.dim * u.size) if want_grad else None
        rc = lib().oracle_rhs(C.byref(self.m), C.byref(self.c), _p(u), _p(dudt),
                              _p(alpha) if alpha is not None else None, _p(lam),
                              _p(grad) if grad is not None else None, self.nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle_rhs failed ({rc})")
        out = {"dudt": dudt, "lambda_max": float(lam[0])}
        if alpha is not None:
            out["alpha"] = alpha
        if grad is not None:
            out["grad"] = grad
        return out

    def step(self, u, dt, scheme=1, nsteps=1, t=0.0):
        u = np.array(u, dtype=np.float64, copy=True)
        rc = lib().oracle_step(C.byref(self.m), C.byref(self.c), _p(u), t, dt, scheme, nsteps,
                               self.nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle_step failed ({rc})")
        return u


# ---------------------------------------------------------------------------
# The same restatement evaluated in x87 long double (liboracle_ld.so, built by
# the Makefile from a copy of prandtl_oracle.cpp with every double lifted):
# the near-exact operator against which both FP64 evaluations, the oracle's and
# the GPU's, are measured when their own rounding of large cancelling terms
# exceeds the 1e-12 budget.
_LD = None
_LDP = C.POINTER(C.c_longdouble)


class _MeshLD(C.Structure):
    _fields_ = [("dim", C.c_int), ("order", C.c_int), ("num_elements", C.c_int), ("num_faces", C.c_int),
                ("elem_adj", _LDP), ("elem_detj", _LDP), ("face_elems", C.POINTER(C.c_int)), ("face_nor", _LDP),
                ("node_adj", _LDP), ("node_detj", _LDP), ("face_node_nor", _LDP)]


class _ConfigLD(C.Structure):
    _fields_ = [("gamma", C.c_longdouble), ("Pr", C.c_longdouble), ("mu", C.c_longdouble),
                ("R_gas", C.c_longdouble), ("alpha_max", C.c_longdouble), ("alpha_min", C.c_longdouble),
                ("parabolic", C.c_int), ("blending", C.c_int), ("sutherland", C.c_int),
                ("quirks", C.c_int), ("surface_dissipation", C.c_int),
                ("num_bcs", C.c_int), ("bcs", C.c_void_p),
                ("axisymmetric", C.c_int), ("node_coords", _LDP), ("axis_rho_floor", C.c_longdouble)]


def lib_ld():
    global _LD
    if _LD is None:
        path = os.path.join(_HERE, "liboracle_ld.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.oracle_rhs.argtypes = [C.POINTER(_MeshLD), C.POINTER(_ConfigLD), _LDP, _LDP, _LDP, _LDP, _LDP, C.c_int]
        L.oracle_rhs.restype = C.c_int
        _LD = L
    return _LD


class LongDoubleOracle:
    """Periodic meshes, planar forms: rhs(u) in long double (u may be float64)."""

    def __init__(self, mesh, gamma=1.4, Pr=0.72, mu=0.02, R_gas=287.05, alpha_max=0.5, alpha_min=0.001,
                 parabolic=0, blending=0, sutherland=0, quirks=0, surface_dissipation=1, nthreads=None):
        ld = np.longdouble
        self.mesh = mesh
        self._adj = np.ascontiguousarray(mesh.elem_adj, dtype=ld)
        self._detj = np.ascontiguousarray(mesh.elem_detj, dtype=ld)
        self._faces = np.ascontiguousarray(mesh.face_elems, dtype=np.int32)
        self._nor = np.ascontiguousarray(mesh.face_nor, dtype=ld)
        self._ngeo = _node_geometry(mesh, ld)
        ng = [a.ctypes.data_as(_LDP) for a in self._ngeo] if self._ngeo else [None, None, None]
        self.m = _MeshLD(mesh.dim, mesh.order, mesh.num_elements, mesh.num_faces,
                         self._adj.ctypes.data_as(_LDP), self._detj.ctypes.data_as(_LDP),
                         self._faces.ctypes.data_as(C.POINTER(C.c_int)), self._nor.ctypes.data_as(_LDP), *ng)
        self.c = _ConfigLD(gamma, Pr, mu, R_gas, alpha_max, alpha_min, parabolic, blending, sutherland, quirks,
                           surface_dissipation, 0, None, 0, None, 0.0)
        self.nthreads = nthreads or os.cpu_count() or 1

    def rhs(self, u, want_alpha=False):
        u = np.ascontiguousarray(u, dtype=np.longdouble)
        dudt = np.empty_like(u)
        alpha = np.empty(self.mesh.num_elements, dtype=np.longdouble) if want_alpha else None
        lam = np.zeros(1, dtype=np.longdouble)
        rc = lib_ld().oracle_rhs(C.byref(self.m), C.byref(self.c), u.ctypes.data_as(_LDP),
                                 dudt.ctypes.data_as(_LDP), alpha.ctypes.data_as(_LDP) if alpha is not None else None,
                                 lam.ctypes.data_as(_LDP), None, self.nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle_rhs (long double) failed ({rc})")
        out = {"dudt": dudt, "lambda_max": lam[0]}
        if alpha is not None:
            out["alpha"] = alpha
        return out


def gl(order):
    n = order + 1
    x, w, D = np.empty(n), np.empty(n), np.empty(n * n)
    lib().oracle_gl(order, _p(x), _p(w), _p(D))
    return x, w, D.reshape(n, n)


# ---------------------------------------------------------------------------
# The reference's own integrator sources, compiled by ref_harness/build_ref.sh
# into _ref/ (only where the reference checkout is present).
_REF_LIBS = {}
_REF_VARIANTS = {(0, 0, 0): "euler", (0, 1, 0): "euler_blend", (1, 0, 0): "ns", (1, 1, 0): "ns_blend",
                 (0, 0, 1): "euler_axi", (0, 1, 1): "euler_blend_axi"}


def ref_available():
    return all(os.path.exists(os.path.join(_HERE, "_ref", f"libref_{v}.so")) for v in _REF_VARIANTS.values())


def build_ref():
    subprocess.run(["bash", os.path.join(_HERE, "ref_harness", "build_ref.sh")], check=True)


def ref_lib(parabolic, blending, axisymmetric=0):
    key = (int(bool(parabolic)), int(bool(blending)), int(bool(axisymmetric)))
    if key not in _REF_LIBS:
        L = C.CDLL(os.path.join(_HERE, "_ref", f"libref_{_REF_VARIANTS[key]}.so"))
        dp = C.POINTER(C.c_double)
        L.ref_rhs.argtypes = [C.POINTER(OracleMesh), C.POINTER(OracleConfig), dp, dp, dp, dp]
        L.ref_rhs.restype = C.c_int
        L.ref_log_mean.argtypes = [C.c_double, C.c_double]
        L.ref_log_mean.restype = C.c_double
        _REF_LIBS[key] = L
    return _REF_LIBS[key]


class RefOperator(Oracle):
    """The reference's DGSEMIntegrator & co. run on the same mesh descriptor.

    Only the reference's own behaviour exists here (no fixed mode); the
    physics switches select the compile-time variant."""

    def rhs(self, u, want_alpha=False, want_grad=False):
        L = ref_lib(self.c.parabolic, self.c.blending, self.c.axisymmetric)
        u = np.ascontiguousarray(u, dtype=np.float64)
        dudt = np.empty_like(u)
        if self.c.axisymmetric:   # the integrators see U recovered from r U (restated in the oracle)
            U = np.empty_like(u)
            if lib().oracle_recover_weighted(C.byref(self.m), C.byref(self.c), _p(u), _p(U)) != 0:
                raise RuntimeError("oracle_recover_weighted failed")
            u = U
        alpha = np.empty(self.mesh.num_elements) if want_alpha else None
        grad = np.empty(self.mesh.dim * u.size) if want_grad else None
        rc = L.ref_rhs(C.byref(self.m), C.byref(self.c), _p(u), _p(dudt),
                       _p(alpha) if alpha is not None else None,
                       _p(grad) if grad is not None else None)
        if rc != 0:
            raise RuntimeError("ref_rhs failed")
        out = {"dudt": dudt}
        if alpha is not None:
            out["alpha"] = alpha
        if grad is not None:
            out["grad"] = grad
        return out


_LSRK_A = (0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
           -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0)
_LSRK_B = (1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
           1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
           2277821191437.0 / 14882151754819.0)


def _ref_step(self, u, dt, scheme=1, nsteps=1, t=0.0):
    """RK steps around the reference RHS: SSP-RK3 in mfem::RK3SSPSolver order
    or Carpenter-Kennedy LSRK4(5) (the reference has no low-storage scheme)."""
    u = np.array(u, dtype=np.float64, copy=True)
    for _ in range(nsteps):
        if scheme == 0:
            k = self.rhs(u)["dudt"]
            y = u + dt * k
            y += dt * self.rhs(y)["dudt"]
            y = 3. / 4 * u + 1. / 4 * y
            y += dt * self.rhs(y)["dudt"]
            u = 1. / 3 * u + 2. / 3 * y
        else:
            du = np.zeros_like(u)
            for a, b in zip(_LSRK_A, _LSRK_B):
                du = a * du + dt * self.rhs(u)["dudt"]
                u = u + b * du
    return u


RefOperator.step = _ref_step
