"""Initial conditions for the benchmark workloads, evaluated at the DG nodes.

States are returned in MFEM ``Ordering::byNODES`` layout:
``u[f*Ndof + e*Np^dim + node]`` with fields (rho, rho*u, rho*v, [rho*w], E).
The reference projects its initial conditions with
``ParGridFunction::ProjectCoefficient`` (``Simulation.cpp:392``), which for a
nodal Gauss-Lobatto L2 space is point evaluation at the nodes, as done here.
"""
from __future__ import annotations

import numpy as np

from .mesh import Mesh, periodic_box


def _pack(rho, mom, E):
    return np.ascontiguousarray(np.concatenate([rho[None], np.asarray(mom), E[None]], axis=0).reshape(-1))


def isentropic_vortex(mesh: Mesh, gamma=1.4, eps=5.0, center=(5.0, 5.0)) -> np.ndarray:
    """Standard isentropic vortex on (rho,u,v,p) = (1,1,1,1)."""
    x, y = mesh.coords[0], mesh.coords[1]
    r2 = (x - center[0]) ** 2 + (y - center[1]) ** 2
    f = np.exp(0.5 * (1.0 - r2))
    u = 1.0 - eps / (2 * np.pi) * f * (y - center[1])
    v = 1.0 + eps / (2 * np.pi) * f * (x - center[0])
    T = 1.0 - (gamma - 1.0) * eps * eps / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho * T
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return _pack(rho, [rho * u, rho * v], E)


def kelvin_helmholtz(mesh: Mesh, gamma=1.4) -> np.ndarray:
    """KelvinHelmholtzInstability.hpp:9-43 (reference IC) on [-1,1]^2."""
    x, y = mesh.coords[0], mesh.coords[1]
    gm1i = 1.0 / (gamma - 1.0)
    B = np.tanh(15.0 * y + 7.5) - np.tanh(15.0 * y - 7.5)
    rho = 0.5 + 0.75 * B
    u = 0.5 * (B - 1.0)
    v = 0.1 * np.sin(2.0 * np.pi * x)
    p = np.ones_like(x)
    E = p * gm1i + rho * 0.5 * (u * u + v * v)
    return _pack(rho, [rho * u, rho * v], E)


def taylor_green(mesh: Mesh, gamma=1.4, mach=0.1) -> np.ndarray:
    """Standard Taylor-Green vortex, isothermal density, on [0, 2pi]^3."""
    x, y, z = mesh.coords
    p0 = 1.0 / (gamma * mach * mach)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    p = p0 + (1.0 / 16.0) * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    rho = p / p0
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return _pack(rho, [rho * u, rho * v, rho * w], E)


def free_stream(mesh: Mesh, gamma=1.4, rho=1.0, vel=None, p=1.0) -> np.ndarray:
    vel = vel if vel is not None else [0.3, -0.2, 0.1][: mesh.dim]
    nn = mesh.ndof
    r = np.full(nn, rho)
    mom = [np.full(nn, rho * v) for v in vel]
    E = np.full(nn, p / (gamma - 1.0) + 0.5 * rho * float(np.dot(vel, vel)))
    return _pack(r, mom, E)


def perturbed(mesh: Mesh, u: np.ndarray, amp=0.05, seed=0) -> np.ndarray:
    """Seeded smooth-plus-noise perturbation that keeps rho, p > 0."""
    rng = np.random.default_rng(seed)
    nf, nn = mesh.num_fields, mesh.ndof
    v = u.reshape(nf, nn).copy()
    rho = v[0] * (1.0 + amp * rng.uniform(-1, 1, nn))
    vel = v[1:1 + mesh.dim] / v[0] + amp * rng.uniform(-1, 1, (mesh.dim, nn))
    gamma = 1.4
    p = (gamma - 1.0) * (v[-1] - 0.5 * v[0] * np.sum((v[1:1 + mesh.dim] / v[0]) ** 2, axis=0))
    p = p * (1.0 + amp * rng.uniform(-1, 1, nn))
    E = p / (gamma - 1.0) + 0.5 * rho * np.sum(vel ** 2, axis=0)
    return _pack(rho, rho * vel, E)


# Workload presets (name -> (mesh factory, IC, physics)).  Sizes follow the
# benchmark configurations: 2D isentropic vortex 32^2 N=3; 3D Taylor-Green
# 32^3 N=3 (Re 1600, Pr 0.71, M 0.1); 2D Kelvin-Helmholtz 256^2 N=3 blended.
def make_case(name: str, n=None, order=3):
    if name == "ivortex":
        m = periodic_box(2, n or 32, order, 0.0, 10.0)
        return m, isentropic_vortex(m), dict(parabolic=0, blending=0)
    if name == "tgv":
        m = periodic_box(3, n or 32, order, 0.0, 2 * np.pi)
        return m, taylor_green(m), dict(parabolic=1, blending=0, mu=1.0 / 1600.0, Pr=0.71)
    if name == "kh":
        m = periodic_box(2, n or 256, order, -1.0, 1.0)
        return m, kelvin_helmholtz(m), dict(parabolic=0, blending=1, alpha_max=0.5)
    raise ValueError(name)


# ---- axisymmetric 15-degree ramp (the reference's TestCases/Euler/2D/Ramp:
# Ramp.hpp RampIC / RampInletBCVector, config.json: AXISYMMETRIC, blending,
# order 1, RK3SSP, dt 1e-4).  In (z, r): [0, 2] x [0, 2], the axis r = 0 for
# z < 1, a 15-degree cone surface from z = 1 to z = 2 (r = 0.26795 there).
RAMP_TAN = 0.26795   # the ramp mesh's end height over its unit length (tan 15 deg)
RAMP_INLET = [1.0, 2.0, 0.0, (1.0 / 1.4) / 0.4 + 0.5 * 1.0 * 2.0 * 2.0]   # rho, rho u, rho v, E (Ma 2)
# boundary-condition table: inlet and top (supersonic inflow of the inlet
# state), outlet (supersonic outflow), axis, ramp (slip wall)
RAMP_BCS = [("state", RAMP_INLET), ("outflow",), ("axis",), ("slip_wall",)]


def ramp_mesh(order=1, nx=98, ny=49) -> Mesh:
    """Structured quadrilaterals of the ramp geometry, uniform in each
    column (the reference's Ramp15deg_v2 mesh has the same 98 x 49 layout,
    graded towards the floor): each column of cells runs from the bottom
    boundary (axis, then ramp) to r = 2, so the cells over the ramp are
    trapezoids, i.e. multilinear elements.  Boundary faces carry the RAMP_BCS
    indices: z = 0 inlet 0, z = 2 outlet 1, bottom axis 2 (z < 1) or ramp 3,
    top 0."""
    def lift(X):   # the box [0,2]^2 mapped onto the ramp domain, r stretched over the floor
        z, r = X[0], X[1]
        floor = np.where(z > 1.0, (z - 1.0) * RAMP_TAN, 0.0)
        return np.stack([np.zeros_like(z), floor * (1.0 - r / 2.0)])
    m = periodic_box(2, (nx, ny), order, (0.0, 0.0), (2.0, 2.0), bcs=[0, 1, 2, 0], warp=lift)
    fe = m.face_elems
    bottom = (fe[:, 2] < 0) & (fe[:, 1] == 2)
    zc = m.coords[0].reshape(m.num_elements, -1).mean(axis=1)
    fe[bottom & (zc[fe[:, 0]] > 1.0), 3] = 3
    return m


def ramp_ic(mesh: Mesh) -> np.ndarray:
    """RampIC (Ramp.hpp): Ma 2 free stream, rho 1, u 2, v 0, p 1/1.4, as the
    axisymmetric RK state r U."""
    nn = mesh.ndof
    U = np.stack([np.full(nn, v) for v in RAMP_INLET])
    return np.ascontiguousarray((U * mesh.coords[1][None, :]).reshape(-1))
