"""CUDA path on meshes read by prandtl_mesh_read, against the oracle (marked gpu).

Read meshes carry re-oriented element frames, Gmsh boundary groups and
Hilbert element orders; the kernels must give the oracle's RHS on the same
descriptor within 1e-12 (per-DOF normalised, FP64).
"""
import os

import numpy as np
import pytest

from conftest import normalized_error
from prandtl_b200.mesh import periodic_box, read_mesh
from test_mesh_io import CAVITY_EULER, CAVITY_NS, MESHES, SHEAR2, smooth_state

pytestmark = pytest.mark.gpu


def _rhs(mesh, u, **kw):
    from prandtl_b200.operator import DGSEMOperator
    op = DGSEMOperator(mesh, **kw)
    d = np.empty_like(u)
    op.Mult(u, d)
    op.close()
    return d


@pytest.mark.parametrize("physics", ["euler", "ns"])
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
@pytest.mark.parametrize("refine,hilbert", [(0, False), (1, True)])
def test_cavity_read_mesh_matches_oracle(oracle_mod, physics, quirks, refine, hilbert):
    m = read_mesh(os.path.join(MESHES, "cavity_6x5.msh"), 3, refine=refine, hilbert=hilbert)
    u = smooth_state(m)
    q = 0 if quirks == "reference" else 1
    if physics == "euler":
        kw = dict(bcs=CAVITY_EULER, blending=1)
    else:
        kw = dict(bcs=CAVITY_NS, parabolic=1, mu=0.01, R_gas=287.05)
    ref = oracle_mod.Oracle(m, quirks=q, **kw).rhs(u)["dudt"]
    kw = {k: (bool(v) if k in ("blending", "parabolic") else v) for k, v in kw.items()}
    got = _rhs(m, u, quirks=quirks, **kw)
    assert normalized_error(got, ref, 4) <= 1e-12


@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_hex_channel_read_mesh_matches_oracle(oracle_mod, quirks):
    m = read_mesh(os.path.join(MESHES, "channel_4x3x2.msh"), 3, hilbert=True)
    u = smooth_state(m)
    q = 0 if quirks == "reference" else 1
    bcs = [("state", [1.3, 0.5, 0.2, -0.1, 2.9]), ("outflow",), ("slip_wall",), ("symmetry",),
           ("pressure_outflow", None, 1.4), ("outflow",)]
    ref = oracle_mod.Oracle(m, quirks=q, bcs=bcs, blending=1).rhs(u)["dudt"]
    assert normalized_error(_rhs(m, u, quirks=quirks, bcs=bcs, blending=True), ref, 5) <= 1e-12
    ns_bcs = [("noslip_adiabatic", dict(wall_vel=[0.0, 0.0, 0.0], heat_flux=0.0)), ("outflow",),
              ("noslip_isothermal", dict(wall_vel=[0.0, 0.0, 0.0], wall_T=0.0045)), ("outflow",),
              ("state", [1.3, 0.5, 0.2, -0.1, 2.9]), ("outflow",)]
    kw = dict(bcs=ns_bcs, mu=0.01, R_gas=287.05)
    ref = oracle_mod.Oracle(m, quirks=q, parabolic=1, **kw).rhs(u)["dudt"]
    assert normalized_error(_rhs(m, u, quirks=quirks, parabolic=True, **kw), ref, 5) <= 1e-12


def test_periodic_read_mesh_equals_generated_box():
    m = read_mesh(os.path.join(MESHES, "periodic_4x3.mesh"), 4)
    b = periodic_box(2, (4, 3), 4, (0.0, 0.0), (2.0, 1.5), affine=SHEAR2)
    u = smooth_state(b)
    kw = dict(parabolic=True, mu=0.01, quirks="fixed")
    assert normalized_error(_rhs(m, u, **kw), _rhs(b, u, **kw), 4) <= 1e-13


BUMP_EULER = [("state", [1.3, 0.5, 0.05, 2.9]), ("outflow",), ("slip_wall",), ("slip_wall",)]
BUMP_NS = [("state", [1.3, 0.5, 0.0, 2.9]), ("outflow",),
           ("noslip_adiabatic", dict(wall_vel=[0.0, 0.0], heat_flux=0.0)),
           ("noslip_isothermal", dict(wall_vel=[0.1, 0.0], wall_T=0.0045))]


@pytest.mark.parametrize("physics", ["euler", "ns"])
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
@pytest.mark.parametrize("refine,hilbert", [(0, False), (1, True)])
def test_bump_channel_multilinear_matches_oracle(oracle_mod, physics, quirks, refine, hilbert):
    """A channel over a bump read from Gmsh (trapezoids, re-oriented frames):
    the per-node geometry kernels against the oracle."""
    m = read_mesh(os.path.join(MESHES, "bump_8x4.msh"), 3, refine=refine, hilbert=hilbert,
                  boundary_conditions={"inlet": 0, "outlet": 1, "floor": 2, "top": 3})
    assert not m.affine
    u = smooth_state(m)
    q = 0 if quirks == "reference" else 1
    if physics == "euler":
        kw = dict(bcs=BUMP_EULER, blending=1)
    else:
        kw = dict(bcs=BUMP_NS, parabolic=1, mu=0.01, R_gas=287.05)
    ref = oracle_mod.Oracle(m, quirks=q, **kw).rhs(u)["dudt"]
    kw = {k: (bool(v) if k in ("blending", "parabolic") else v) for k, v in kw.items()}
    assert normalized_error(_rhs(m, u, quirks=quirks, **kw), ref, 4) <= 1e-12


@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_warped_hex_box_multilinear_matches_oracle(oracle_mod, quirks):
    m = read_mesh(os.path.join(MESHES, "warped_3x3x2.msh"), 2, hilbert=True)
    assert not m.affine
    u = smooth_state(m)
    q = 0 if quirks == "reference" else 1
    bcs = [("state", [1.3, 0.5, 0.2, -0.1, 2.9]), ("outflow",), ("slip_wall",), ("symmetry",),
           ("pressure_outflow", None, 1.4), ("outflow",)]
    ref = oracle_mod.Oracle(m, quirks=q, bcs=bcs, blending=1).rhs(u)["dudt"]
    assert normalized_error(_rhs(m, u, quirks=quirks, bcs=bcs, blending=True), ref, 5) <= 1e-12
    ns_bcs = [("noslip_adiabatic", dict(wall_vel=[0.0, 0.0, 0.0], heat_flux=0.0)), ("outflow",),
              ("noslip_isothermal", dict(wall_vel=[0.0, 0.0, 0.0], wall_T=0.0045)), ("outflow",),
              ("state", [1.3, 0.5, 0.2, -0.1, 2.9]), ("outflow",)]
    kw = dict(bcs=ns_bcs, mu=0.01, R_gas=287.05)
    ref = oracle_mod.Oracle(m, quirks=q, parabolic=1, **kw).rhs(u)["dudt"]
    assert normalized_error(_rhs(m, u, quirks=quirks, parabolic=True, **kw), ref, 5) <= 1e-12
