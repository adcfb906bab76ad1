"""Python mirror of the reference operator interface, backed by the C ABI.

``DGSEMOperator`` mirrors ``Prandtl::DGSEMOperator`` (src/Operators/DGSEMOperator.hpp:15-141):
``Mult(u, dudt)`` evaluates the DGSEM right-hand side, ``GetMaxCharSpeed()``
returns the largest characteristic speed seen by the last evaluation, and the
time lives in ``t`` (TimeDependentOperator::SetTime / GetTimeRef).  ``Step``
plays the role of the mfem::ODESolver the reference drives it with
(Simulation.cpp:177-206, :1010).

Arrays may be numpy (host memory: staged through the handle's device buffers)
or torch CUDA tensors (device memory: zero copy).  Every call goes to the
CUDA kernels; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh

_SCHEMES = {"RK3SSP": _lib.RK3SSP, "LSRK45": _lib.LSRK45, 0: _lib.RK3SSP, 1: _lib.LSRK45}


def _ptr(a):
    """(pointer, flag) for a numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("arrays must be C-contiguous float64")
        return a.ctypes.data, _lib.PTR_HOST
    if hasattr(a, "data_ptr"):   # torch.Tensor
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("tensors must be contiguous float64")
        return a.data_ptr(), (_lib.PTR_DEVICE if a.is_cuda else _lib.PTR_HOST)
    raise TypeError(f"unsupported array type {type(a)}")


class MeshArrays:
    """The C-ABI mesh descriptor of a Mesh, with the arrays it points into kept alive."""

    def __init__(self, mesh: Mesh):
        self.adj = np.ascontiguousarray(mesh.elem_adj, dtype=np.float64)
        self.detj = np.ascontiguousarray(mesh.elem_detj, dtype=np.float64)
        self.faces = np.ascontiguousarray(mesh.face_elems, dtype=np.int32)
        self.nor = np.ascontiguousarray(mesh.face_nor, dtype=np.float64)
        dp = C.POINTER(C.c_double)
        # non-affine elements: per-node transformation and per-face-node normals
        self.node = None if mesh.affine else tuple(
            np.ascontiguousarray(a, dtype=np.float64) for a in (mesh.node_adj, mesh.node_detj, mesh.face_node_nor))
        ng = [a.ctypes.data_as(dp) for a in self.node] if self.node else [None, None, None]
        self.desc = _lib.MeshDesc(mesh.dim, mesh.order, mesh.num_elements, mesh.num_faces,
                                  self.adj.ctypes.data_as(dp), self.detj.ctypes.data_as(dp),
                                  self.faces.ctypes.data_as(C.POINTER(C.c_int)),
                                  self.nor.ctypes.data_as(dp), *ng)


def make_bcs(bcs):
    """ctypes array of prandtl_bc from [(type name, state or None, p or None), ...]:
    type names "state", "outflow", "slip_wall", "symmetry", "pressure_outflow",
    "riemann" (state = outer primitive state), "inflow_rv" (state = rho, V) and
    "inflow_pttt" (second item a dict of pt, Tt, cp, theta, phi), "noslip_adiabatic"
    (dict of wall_vel, heat_flux) and "noslip_isothermal" (dict of wall_vel, wall_T)."""
    if not bcs:
        return None
    arr = (_lib.BC * len(bcs))()
    for k, b in enumerate(bcs):
        kind, state, p = (tuple(b) + (None, None))[:3]
        arr[k].type = _lib.BC_TYPES[kind]
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


def make_config(*, gamma=1.4, Pr=0.72, mu=0.02, R_gas=287.05, parabolic=False, blending=False,
                sutherland=False, alpha_max=0.5, alpha_min=0.001, quirks="reference",
                surface_dissipation=True, precision="fp64", timeout_s=120.0, bcs=None,
                axisymmetric=False, node_coords=None, axis_rho_floor=0.0) -> _lib.Config:
    """prandtl_config from the DGSEMOperator keyword arguments (the BC array
    and the axisymmetric node coordinates are kept alive on the returned
    object)."""
    cfg = _lib.Config()
    _lib.load().prandtl_config_default(C.byref(cfg))
    cfg.gamma, cfg.Pr, cfg.mu, cfg.R_gas = gamma, Pr, mu, R_gas
    cfg.alpha_max, cfg.alpha_min = alpha_max, alpha_min
    cfg.parabolic, cfg.blending, cfg.sutherland = int(parabolic), int(blending), int(sutherland)
    if quirks not in ("reference", "fixed", 0, 1):
        raise ValueError("quirks must be 'reference' or 'fixed'")
    cfg.quirks = 1 if quirks in ("fixed", 1) else 0
    cfg.surface_dissipation = int(bool(surface_dissipation))
    if precision not in ("fp64", "fp32"):
        raise ValueError("precision must be 'fp64' or 'fp32' (FP32 bulk, FP64 RK state)")
    cfg.precision = 1 if precision == "fp32" else 0
    cfg.timeout_s = timeout_s
    cfg._bcs = make_bcs(bcs)
    cfg.num_bcs = len(bcs) if bcs else 0
    cfg.bcs = cfg._bcs
    cfg.axisymmetric = int(bool(axisymmetric))
    cfg.axis_rho_floor = float(axis_rho_floor)
    if axisymmetric and node_coords is not None:
        cfg._xy = np.ascontiguousarray(node_coords, dtype=np.float64)
        cfg.node_coords = cfg._xy.ctypes.data_as(C.POINTER(C.c_double))
    return cfg


class DGSEMOperator:
    def __init__(self, mesh: Mesh, *, gamma=1.4, Pr=0.72, mu=0.02, R_gas=287.05,
                 parabolic=False, blending=False, sutherland=False, alpha_max=0.5,
                 alpha_min=0.001, quirks="reference", surface_dissipation=True,
                 precision="fp64", timeout_s=120.0, bcs=None, axisymmetric=False, axis_rho_floor=0.0):
        """axisymmetric: the reference's AXISYMMETRIC build -- 2D Euler in
        (z, r) = (x, y); Mult takes and returns the r-weighted state r U.
        axis_rho_floor: density floor of its axis reconstruction (0: 1e-12)."""
        L = _lib.load()
        self.mesh = mesh
        self._arrays = MeshArrays(mesh)
        desc = self._arrays.desc
        cfg = make_config(gamma=gamma, Pr=Pr, mu=mu, R_gas=R_gas, parabolic=parabolic,
                          blending=blending, sutherland=sutherland, alpha_max=alpha_max,
                          alpha_min=alpha_min, quirks=quirks, surface_dissipation=surface_dissipation,
                          precision=precision, timeout_s=timeout_s, bcs=bcs,
                          axisymmetric=axisymmetric, node_coords=mesh.coords if axisymmetric else None,
                          axis_rho_floor=axis_rho_floor)
        h = C.c_void_p()
        _lib.check(L.prandtl_create(C.byref(desc), C.byref(cfg), C.byref(h)), None)
        self._h = h
        self._L = L
        self.t = 0.0
        self.max_char_speed = -1.0
        self.height = self.width = mesh.num_fields * mesh.ndof

    # -- mfem::TimeDependentOperator surface
    def SetTime(self, t: float):
        self.t = float(t)

    def GetTime(self) -> float:
        return self.t

    def Mult(self, u, dudt):
        pu, fu = _ptr(u)
        pd, fd = _ptr(dudt)
        if fu != fd:
            raise ValueError("u and dudt must both be host or both be device arrays")
        lam = C.c_double(0.0)
        _lib.check(self._L.prandtl_rhs(self._h, pu, pd, self.t, C.byref(lam), fu), self._h)
        self.max_char_speed = lam.value
        return dudt

    def GetMaxCharSpeed(self) -> float:
        return self.max_char_speed

    # -- mfem::ODESolver::Step equivalent
    def Step(self, u, dt: float, scheme="RK3SSP", nsteps=1):
        pu, fu = _ptr(u)
        _lib.check(self._L.prandtl_step(self._h, pu, self.t, float(dt), _SCHEMES[scheme],
                                        int(nsteps), fu), self._h)
        self.t += nsteps * dt
        return u

    def alpha(self) -> np.ndarray:
        out = np.empty(self.mesh.num_elements)
        _lib.check(self._L.prandtl_get_alpha(self._h, out.ctypes.data, _lib.PTR_HOST), self._h)
        return out

    def recover_state(self, rU, U=None):
        """Axisymmetric form: the conserved U that the fluxes see, recovered
        from the r-weighted state rU (the reference writes its output fields
        from this U)."""
        if U is None:
            if isinstance(rU, np.ndarray):
                U = np.empty_like(rU)
            else:
                import torch
                U = torch.empty_like(rU)
        pr, fr = _ptr(rU)
        pU, fU = _ptr(U)
        if fr != fU:
            raise ValueError("rU and U must both be host or both be device arrays")
        _lib.check(self._L.prandtl_recover_state(self._h, pr, pU, fr), self._h)
        return U

    def budgets(self, u, dudt=None) -> dict:
        """FP64 integrals over the mesh, reduced on the device: the conserved
        fields, the entropy function -rho s / (gamma - 1), and with dudt their
        rates and the entropy production (integral of v . dudt)."""
        pu, fu = _ptr(u)
        pd = None
        if dudt is not None:
            pd, fd = _ptr(dudt)
            if fd != fu:
                raise ValueError("u and dudt must both be host or both be device arrays")
        nf = self.mesh.num_fields
        out = np.zeros(2 * nf + 2)
        _lib.check(self._L.prandtl_budgets(self._h, pu, pd, out.ctypes.data, fu), self._h)
        return {"conserved": out[:nf].copy(), "entropy": float(out[nf]),
                "rates": out[nf + 1:2 * nf + 1].copy(), "entropy_rate": float(out[2 * nf + 1])}

    def cfl_dt(self, cfl: float, lambda_max: float | None = None) -> float:
        lam = self.max_char_speed if lambda_max is None else lambda_max
        return self._L.prandtl_cfl_dt(cfl, self.mesh.hmin, lam, self.mesh.order)

    def set_stream(self, stream_ptr: int):
        _lib.check(self._L.prandtl_set_stream(self._h, C.c_void_p(stream_ptr)), self._h)

    def synchronize(self):
        _lib.check(self._L.prandtl_synchronize(self._h), self._h)

    def profile(self, enable: bool = True):
        """Bracket every kernel launch with CUDA events (instrumentation)."""
        _lib.check(self._L.prandtl_profile(self._h, int(enable)), self._h)

    def profile_reset(self):
        _lib.check(self._L.prandtl_profile_reset(self._h), self._h)

    def profile_read(self):
        """{kernel name: (total device ms, launches)} since the last reset."""
        out = {}
        for name, k in (("rhs", _lib.KERNEL_RHS), ("lift", _lib.KERNEL_LIFT)):
            ms, n = C.c_double(0.0), C.c_longlong(0)
            _lib.check(self._L.prandtl_profile_read(self._h, k, C.byref(ms), C.byref(n)), self._h)
            out[name] = (ms.value, n.value)
        return out

    @property
    def kernel_launches(self) -> int:
        return int(self._L.prandtl_kernel_launches(self._h))

    @property
    def device_bytes(self) -> int:
        return int(self._L.prandtl_device_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.prandtl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
