"""Generate golden RHS vectors from the reference's own DGSEM sources.

Runs oracle/_ref/libref_*.so (the reference's DGSEMIntegrator, LiftingBR1,
ChandrashekarFlux, NavierStokesFlux, BasicOperations, PerssonPeraireIndicator,
ModalBasis and boundary integrators compiled unmodified by
oracle/ref_harness/build_ref.sh) on small seeded cases and stores inputs and
outputs in reference_rhs.npz.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from prandtl_b200 import cases  # noqa: E402
from prandtl_b200.mesh import periodic_box  # noqa: E402

# (name, dim, n, order, parabolic, blending, amplitude, seed)
CASES = [
    ("euler2d_n3_N3", 2, 3, 3, 0, 0, 0.10, 1),
    ("euler2d_blend_n3_N3", 2, 3, 3, 0, 1, 0.30, 2),
    ("ns2d_n3_N2", 2, 3, 2, 1, 0, 0.10, 3),
    ("ns2d_blend_n2_N4", 2, 2, 4, 1, 1, 0.30, 4),
    ("euler3d_n2_N2", 3, 2, 2, 0, 0, 0.10, 5),
    ("euler3d_blend_n2_N3", 3, 2, 3, 0, 1, 0.30, 6),
    ("ns3d_n2_N3", 3, 2, 3, 1, 0, 0.10, 7),
    ("ns3d_blend_n2_N2", 3, 2, 2, 1, 1, 0.30, 8),
]
PHYS = dict(gamma=1.4, Pr=0.71, mu=0.01, R_gas=287.05, alpha_max=0.5, alpha_min=0.001)

# Euler with boundary faces: (name, dim, n, order, blending, amplitude, seed);
# every case uses BCS, the sides of SIDES[dim] (2*dir + side -> BCS index).
BOUNDARY_CASES = [
    ("euler2d_bdr_n3_N3", 2, 3, 3, 0, 0.10, 11),
    ("euler2d_bdr_blend_n3_N2", 2, 3, 2, 1, 0.30, 12),
    ("euler3d_bdr_n2_N3", 3, 2, 3, 0, 0.10, 13),
    ("euler3d_bdr_blend_n2_N2", 3, 2, 2, 1, 0.30, 14),
]
BCS = {2: [("state", [1.3, 0.5, 0.2, 2.9]), ("outflow",), ("slip_wall",), ("symmetry",), ("pressure_outflow", None, 1.4)],
       3: [("state", [1.3, 0.5, 0.2, -0.1, 2.9]), ("outflow",), ("slip_wall",), ("symmetry",),
           ("pressure_outflow", None, 1.4)]}
SIDES = {2: [0, 4, 2, 3], 3: [0, 1, 2, 3, 4, 2]}

# Characteristic and subsonic-inflow conditions, same case format (CHAR_BCS on
# the sides CHAR_SIDES).  The reference's SubsonicInflowPtTtAng constructor
# writes past its direction vector in 3D, so 3D cases leave it out.
PTTT = ("inflow_pttt", dict(pt=1.7, Tt=1.3, cp=3.5, theta=20.0, phi=70.0))
CHAR_CASES = [
    ("euler2d_char_n3_N3", 2, 3, 3, 0, 0.10, 21),
    ("euler2d_char_blend_n2_N4", 2, 2, 4, 1, 0.30, 22),
    ("euler3d_char_n2_N2", 3, 2, 2, 0, 0.10, 23),
    ("euler3d_char_blend_n2_N3", 3, 2, 3, 1, 0.30, 24),
]
CHAR_BCS = {2: [("riemann", [1.25, 0.35, -0.1, 1.6]), ("inflow_rv", [1.15, 0.45, -0.25]), PTTT,
                ("riemann", [1.2, 1.8, 0.1, 1.5]), ("outflow",)],
            3: [("riemann", [1.25, 0.35, -0.1, 0.05, 1.6]), ("inflow_rv", [1.15, 0.45, -0.25, 0.15]),
                ("riemann", [1.2, 1.8, 0.1, 0.0, 1.5]), ("outflow",)]}
CHAR_SIDES = {2: [1, 0, 2, 3], 3: [1, 0, 2, 3, 0, 2]}

# Navier-Stokes with boundary faces (parabolic = 1): no-slip walls (a moving
# adiabatic lid with a heat flux, an isothermal wall), outflow and the
# inflow/outflow types whose viscous boundary flux vanishes.  Slip wall,
# symmetry and pt/Tt inflow have no viscous treatment in the reference, and its
# Riemann-invariant lifting reads an unset face normal (NaN here), so the
# golden cases leave those out.
NS_BCS = {d: [("noslip_adiabatic", dict(wall_vel=[0.3, 0.0, 0.1][:d], heat_flux=0.01)),
              ("noslip_isothermal", dict(wall_vel=[0.0, 0.05, 0.0][:d], wall_T=0.0045)),
              ("outflow",),
              ("state", [1.3, 0.5, 0.2, 2.9] if d == 2 else [1.3, 0.5, 0.2, -0.1, 2.9]),
              ("pressure_outflow", None, 1.4),
              ("riemann", [1.25, 0.35, -0.1, 1.6] if d == 2 else [1.25, 0.35, -0.1, 0.05, 1.6]),
              ("inflow_rv", [1.15, 0.45, -0.25, 0.15][: d + 1])] for d in (2, 3)}
NS_WALL_SIDES = {2: [3, 2, 1, 0], 3: [3, 2, 1, 0, 0, 1]}
NS_CHAR_SIDES = {2: [2, 4, 6, 0], 3: [2, 4, 6, 0, 1, 3]}
NS_WALL_CASES = [
    ("ns2d_walls_n3_N3", 2, 3, 3, 0, 0.10, 31),
    ("ns2d_walls_blend_n2_N4", 2, 2, 4, 1, 0.30, 32),
    ("ns3d_walls_n2_N2", 3, 2, 2, 0, 0.10, 33),
    ("ns3d_walls_blend_n2_N3", 3, 2, 3, 1, 0.30, 34),
]
NS_CHAR_CASES = [
    ("ns2d_char_n3_N2", 2, 3, 2, 0, 0.10, 41),
    ("ns3d_char_n2_N3", 3, 2, 3, 1, 0.30, 42),
]
# name -> (cases, BC tables, sides, parabolic)
BC_SETS = {"walls": (BOUNDARY_CASES, BCS, SIDES, 0), "char": (CHAR_CASES, CHAR_BCS, CHAR_SIDES, 0),
           "ns_walls": (NS_WALL_CASES, NS_BCS, NS_WALL_SIDES, 1),
           "ns_char": (NS_CHAR_CASES, NS_BCS, NS_CHAR_SIDES, 1)}


# Axisymmetric (z, r) Euler (the reference built with AXISYMMETRIC): state r U
# on a sheared box over 0 <= r <= 1 with the axis at r = 0;
# (name, n, order, blending, amplitude, seed).
AXI_BCS = [("state", [1.3, 0.5, 0.0, 2.9]), ("outflow",), ("axis",), ("slip_wall",)]
AXI_SIDES = [0, 1, 2, 3]
AXI_CASES = [
    ("axi2d_n4x3_N1", (4, 3), 1, 0, 0.10, 31),
    ("axi2d_n4x3_N3", (4, 3), 3, 0, 0.10, 32),
    ("axi2d_blend_n4x3_N2", (4, 3), 2, 1, 0.30, 33),
    ("axi2d_blend_n3x2_N4", (3, 2), 4, 1, 0.30, 34),
]


def axi_inputs(n, order, blending, amp, seed):
    mesh = periodic_box(2, n, order, (0.0, 0.0), (2.0, 1.0), bcs=AXI_SIDES,
                        affine=np.array([[1.0, 0.1], [0.0, 1.0]]))
    U = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.2, vel=[0.3, 0.05], p=1.5),
                        amp=amp, seed=seed).reshape(4, -1)
    return mesh, (U * mesh.coords[1][None, :]).reshape(-1)


# Non-affine (multilinear) elements: the box's element corners moved by a
# smooth displacement (periodic on the unit box), so every element is a
# general bilinear quadrilateral / trilinear hexahedron with per-node metrics;
# (name, dim, n, order, parabolic, blending, amplitude, seed, boundary set or None).
CURVED_CASES = [
    ("curved_euler2d_blend_n3_N3", 2, 3, 3, 0, 1, 0.30, 51, None),
    ("curved_euler2d_n3_N1", 2, 3, 1, 0, 0, 0.10, 52, None),
    ("curved_ns2d_n3_N2", 2, 3, 2, 1, 0, 0.10, 53, None),
    ("curved_euler3d_n3_N2", 3, 3, 2, 0, 0, 0.10, 54, None),
    ("curved_ns3d_blend_n3_N2", 3, 3, 2, 1, 1, 0.30, 55, None),
    ("curved_euler2d_bdr_blend_n3_N2", 2, 3, 2, 0, 1, 0.30, 56, "walls"),
    ("curved_ns2d_walls_n3_N3", 2, 3, 3, 1, 0, 0.10, 57, "ns_walls"),
    ("curved_euler3d_char_n3_N2", 3, 3, 2, 0, 0, 0.10, 58, "char"),
]
CURVED_AXI_CASES = [
    ("curved_axi2d_n4x3_N1", (4, 3), 1, 0, 0.10, 61),
    ("curved_axi2d_blend_n4x3_N2", (4, 3), 2, 1, 0.30, 62),
]


def warp_field(dim, amp):
    """Corner displacement on the unit box, periodic in every direction."""
    def w(X):
        s = [np.sin(2 * np.pi * X[d]) for d in range(dim)]
        c = [np.cos(2 * np.pi * X[d]) for d in range(dim)]
        if dim == 2:
            return amp * np.stack([s[1] * (0.6 + 0.4 * s[0]), s[0] * (0.5 + 0.5 * c[1])])
        return amp * np.stack([s[1] * s[2] + 0.3 * s[0] * c[1], s[0] * s[2] + 0.3 * s[1] * c[2],
                               s[0] * s[1] + 0.3 * s[2] * c[0]])
    return w


def axi_warp(X):
    """Displacement of the (z, r) box [0,2] x [0,1] that keeps the axis r = 0 and
    the other sides straight."""
    z, r = X[0], X[1]
    return np.stack([0.06 * np.sin(np.pi * r) * np.sin(np.pi * z), 0.05 * np.sin(np.pi * r) * np.sin(0.5 * np.pi * z)])


def curved_inputs(dim, n, order, amp, seed, bset=None):
    sides = BC_SETS[bset][2][dim] if bset else None
    mesh = periodic_box(dim, n, order, 0.0, 1.0, bcs=sides, warp=warp_field(dim, 0.06))
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5)
    return mesh, cases.perturbed(mesh, base, amp=amp, seed=seed)


def curved_axi_inputs(n, order, blending, amp, seed):
    mesh = periodic_box(2, n, order, (0.0, 0.0), (2.0, 1.0), bcs=AXI_SIDES, warp=axi_warp)
    U = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.2, vel=[0.3, 0.05], p=1.5),
                        amp=amp, seed=seed).reshape(4, -1)
    return mesh, (U * mesh.coords[1][None, :]).reshape(-1)


def bc_example(kind, dim):
    """One condition of the given type with constant data for a dim-D case;
    "riemann_supersonic" is the Riemann condition with a supersonic outer state."""
    if kind == "riemann_supersonic":
        return CHAR_BCS[dim][2 if dim == 3 else 3]
    for bcs in (BCS[dim], CHAR_BCS[dim], [PTTT], NS_BCS[dim]):
        for b in bcs:
            if b[0] == kind:
                return b
    raise KeyError(kind)


def case_inputs(dim, n, order, amp, seed, bcs=None):
    rng = np.random.default_rng(100 + seed)
    A = np.eye(dim) + 0.15 * rng.uniform(-1, 1, (dim, dim))
    mesh = periodic_box(dim, n, order, 0.0, 1.0, affine=A, bcs=bcs)
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5)
    return mesh, A, cases.perturbed(mesh, base, amp=amp, seed=seed)


def main():
    import pyoracle
    if not pyoracle.ref_available():
        pyoracle.build_ref()
    out = {}
    for name, dim, n, order, par, bl, amp, seed in CASES:
        mesh, A, u = case_inputs(dim, n, order, amp, seed)
        r = pyoracle.RefOperator(mesh, parabolic=par, blending=bl, **PHYS).rhs(u, want_alpha=True)
        out[f"{name}/affine"] = A
        out[f"{name}/u"] = u
        out[f"{name}/dudt"] = r["dudt"]
        out[f"{name}/alpha"] = r["alpha"]
    for bcases, bcs, sides, par in BC_SETS.values():
        for name, dim, n, order, bl, amp, seed in bcases:
            mesh, A, u = case_inputs(dim, n, order, amp, seed, bcs=sides[dim])
            r = pyoracle.RefOperator(mesh, parabolic=par, blending=bl, bcs=bcs[dim], **PHYS).rhs(u, want_alpha=True)
            out[f"{name}/affine"] = A
            out[f"{name}/u"] = u
            out[f"{name}/dudt"] = r["dudt"]
            out[f"{name}/alpha"] = r["alpha"]
    for name, n, order, bl, amp, seed in AXI_CASES:
        mesh, u = axi_inputs(n, order, bl, amp, seed)
        r = pyoracle.RefOperator(mesh, blending=bl, bcs=AXI_BCS, axisymmetric=1).rhs(u, want_alpha=True)
        out[f"{name}/u"] = u
        out[f"{name}/dudt"] = r["dudt"]
        out[f"{name}/alpha"] = r["alpha"]
    for name, dim, n, order, par, bl, amp, seed, bset in CURVED_CASES:
        mesh, u = curved_inputs(dim, n, order, amp, seed, bset)
        bcs = BC_SETS[bset][1][dim] if bset else None
        r = pyoracle.RefOperator(mesh, parabolic=par, blending=bl, bcs=bcs, **PHYS).rhs(u, want_alpha=True)
        out[f"{name}/u"] = u
        out[f"{name}/dudt"] = r["dudt"]
        out[f"{name}/alpha"] = r["alpha"]
    for name, n, order, bl, amp, seed in CURVED_AXI_CASES:
        mesh, u = curved_axi_inputs(n, order, bl, amp, seed)
        r = pyoracle.RefOperator(mesh, blending=bl, bcs=AXI_BCS, axisymmetric=1).rhs(u, want_alpha=True)
        out[f"{name}/u"] = u
        out[f"{name}/dudt"] = r["dudt"]
        out[f"{name}/alpha"] = r["alpha"]
    np.savez_compressed(os.path.join(HERE, "reference_rhs.npz"), **out)
    print(f"wrote {len(CASES) + sum(len(v[0]) for v in BC_SETS.values()) + len(AXI_CASES)+ len(CURVED_CASES) + len(CURVED_AXI_CASES)} cases")


if __name__ == "__main__":
    main()
