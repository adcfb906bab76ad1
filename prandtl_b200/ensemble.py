"""Seeded synthetic workloads for the batch and serving forms.

``tgv_ensemble``: independent 3D Navier-Stokes Taylor-Green vortices of
uneven sizes.  Elements per direction n ~ U{4..16} (n^3 hexes on [0,2pi]^3),
order N ~ U{2,3,4,5}, Mach ~ U[0.05,0.3] and Re ~ logU[100,3200], drawn from
numpy PCG64.

``serving_stream``: Poisson arrivals of solve requests.  Half are 2D Euler
isentropic vortices (n ~ U{16..128} squared, N in {3,4}); half are 3D TGVs
(n ~ U{8..24} cubed, N in {2,3}).  Each runs steps ~ U{50..500}.

The time step is fixed per solve: dt = cfl*hmin/(lambda0 (N+1)^2), where
lambda0 = max |V|+c of the initial state.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import cases
from .mesh import Mesh, periodic_box

TWO_PI = 2.0 * math.pi
_MESHES: dict = {}


@dataclasses.dataclass
class Member:
    kind: str            # "tgv" (3D Navier-Stokes) or "ivortex" (2D Euler)
    n: int               # elements per direction
    order: int
    mach: float = 0.1
    re: float = 1600.0
    nsteps: int = 100
    arrival: float = 0.0  # seconds after the stream starts (serving)

    def mesh(self) -> Mesh:
        key = (self.kind, self.n, self.order)
        if key not in _MESHES:   # meshes are read-only; members of one shape share one
            if self.kind == "tgv":
                _MESHES[key] = periodic_box(3, self.n, self.order, 0.0, TWO_PI)
            else:
                _MESHES[key] = periodic_box(2, self.n, self.order, 0.0, 10.0)
        return _MESHES[key]

    def physics(self) -> dict:
        if self.kind == "tgv":
            return dict(parabolic=True, mu=1.0 / self.re, Pr=0.71, quirks="fixed")
        return dict(quirks="fixed")

    def initial_state(self, mesh: Mesh) -> np.ndarray:
        if self.kind == "tgv":
            return cases.taylor_green(mesh, mach=self.mach)
        return cases.isentropic_vortex(mesh)

    def nodes(self) -> int:
        d = 3 if self.kind == "tgv" else 2
        return (self.n * (self.order + 1)) ** d

    def dofs(self) -> int:
        return self.nodes() * (5 if self.kind == "tgv" else 4)


def max_char_speed(u: np.ndarray, dim: int, gamma: float = 1.4) -> float:
    """max |V| + c over the nodes of a byNODES state."""
    q = u.reshape(dim + 2, -1)
    rho = q[0]
    v2 = sum((q[1 + d] / rho) ** 2 for d in range(dim))
    p = (gamma - 1.0) * (q[dim + 1] - 0.5 * rho * v2)
    return float(np.max(np.sqrt(v2) + np.sqrt(gamma * p / rho)))


def fixed_dt(mesh: Mesh, u0: np.ndarray, cfl: float) -> float:
    lam = max_char_speed(u0, mesh.dim)
    return cfl * mesh.hmin / (lam * (mesh.order + 1) ** 2)


def tgv_ensemble(count=512, seed=20261203, n_range=(4, 16), orders=(2, 3, 4, 5),
                 mach=(0.05, 0.3), re=(100.0, 3200.0), nsteps=100):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        order = int(orders[int(rng.integers(0, len(orders)))])
        m = float(rng.uniform(*mach))
        r = float(math.exp(rng.uniform(math.log(re[0]), math.log(re[1]))))
        out.append(Member("tgv", n, order, m, r, nsteps))
    return out


def serving_stream(count=10000, seed=20261204, rate=1.0, iv_n=(16, 128), iv_orders=(3, 4),
                   tgv_n=(8, 24), tgv_orders=(2, 3), steps=(50, 500)):
    """Requests with Poisson arrival times at `rate` per second."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate))
        if rng.uniform() < 0.5:
            m = Member("ivortex", int(rng.integers(iv_n[0], iv_n[1] + 1)),
                       int(iv_orders[int(rng.integers(0, len(iv_orders)))]))
        else:
            m = Member("tgv", int(rng.integers(tgv_n[0], tgv_n[1] + 1)),
                       int(tgv_orders[int(rng.integers(0, len(tgv_orders)))]))
        m.nsteps = int(rng.integers(steps[0], steps[1] + 1))
        m.arrival = t
        out.append(m)
    return out
