"""Euler boundary faces on the GPU against the oracle and the reference's own
boundary-condition sources (marked gpu).

A boundary face {elem1, lface1, -1, bc} takes its numerical flux from the BC
table entry bc: a specified outer state (Rusanov), supersonic outflow, slip
wall, symmetry plane or subsonic pressure outflow.  Tolerances as for the
periodic parity tests: per-DOF normalised error <= 1e-12 for one RHS in FP64,
<= 1e-10 for trajectories; FP32 bulk within 2e-3 relative L2 of FP64 for one
RHS; batches within 1e-12 of the one-operator path in FP64.
"""
import os
import sys

import numpy as np
import pytest

from conftest import normalized_error
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
TRAJ_TOL = 1e-10
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

BCS = make_golden.BCS
SIDES = make_golden.SIDES


def _op(mesh, **kw):
    from prandtl_b200.operator import DGSEMOperator
    return DGSEMOperator(mesh, **kw)


def _affine(dim, seed=1):
    rng = np.random.default_rng(seed)
    return np.eye(dim) + 0.15 * rng.uniform(-1, 1, (dim, dim))


def test_boundary_rhs_matches_reference_golden():
    gold = np.load(os.path.join(HERE, "golden", "reference_rhs.npz"))
    for bcases, bcs, sides, par in make_golden.BC_SETS.values():
        for name, dim, n, order, bl, amp, seed in bcases:
            mesh, A, u = make_golden.case_inputs(dim, n, order, amp, seed, bcs=sides[dim])
            op = _op(mesh, parabolic=bool(par), blending=bool(bl), quirks="reference", bcs=bcs[dim],
                     **make_golden.PHYS)
            d = np.empty_like(u)
            op.Mult(u, d)
            err = normalized_error(d, gold[f"{name}/dudt"], mesh.num_fields)
            assert err <= RHS_TOL, f"{name}: {err:.3e}"
            np.testing.assert_allclose(op.alpha(), gold[f"{name}/alpha"], rtol=0, atol=1e-12)
            op.close()


@pytest.mark.parametrize("dim,n,order", [(2, 3, 1), (2, 3, 2), (2, 2, 3), (2, 2, 4), (2, 2, 5),
                                         (3, 2, 1), (3, 2, 2), (3, 2, 3), (3, 2, 4), (3, 1, 5)])
@pytest.mark.parametrize("blending", [0, 1])
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
@pytest.mark.parametrize("bset", ["walls", "char", "ns_walls", "ns_char"])
def test_boundary_rhs_matches_oracle(oracle_mod, dim, n, order, blending, quirks, bset):
    _, bcs, sides, par = make_golden.BC_SETS[bset]
    bcs = bcs[dim] + ([make_golden.PTTT] if dim == 3 and bset == "char" else [])
    sides = list(sides[dim])
    if dim == 3 and bset == "char":
        sides[3] = len(bcs) - 1   # 3D inflow_pttt (direction cos f, checked against the oracle only)
    if bset == "ns_char" and quirks == "fixed":
        sides[0] = 5   # Riemann invariants (defined in the Navier-Stokes form with quirks fixed)
    mesh = periodic_box(dim, n, order, 0.0, 1.0, affine=_affine(dim, order), bcs=sides)
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5)
    u = cases.perturbed(mesh, base, amp=0.3 if blending else 0.1, seed=order + 7 * dim)
    q = 0 if quirks == "reference" else 1
    kw = dict(parabolic=par, blending=blending, bcs=bcs, **(make_golden.PHYS if par else {}))
    ref = oracle_mod.Oracle(mesh, quirks=q, **kw).rhs(u, want_alpha=True)
    kw["parabolic"], kw["blending"] = bool(par), bool(blending)
    op = _op(mesh, quirks=quirks, **kw)
    d = np.empty_like(u)
    op.Mult(u, d)
    err = normalized_error(d, ref["dudt"], mesh.num_fields)
    assert err <= RHS_TOL, f"normalised error {err:.3e}"
    assert abs(op.GetMaxCharSpeed() - ref["lambda_max"]) <= 1e-13 * ref["lambda_max"]
    if blending:
        np.testing.assert_allclose(op.alpha(), ref["alpha"], rtol=0, atol=1e-12)
    op.close()


@pytest.mark.parametrize("kind", ["state", "outflow", "slip_wall", "symmetry", "pressure_outflow", "riemann",
                                  "riemann_supersonic", "inflow_rv", "inflow_pttt"])
def test_each_boundary_type_alone(oracle_mod, kind):
    """Every side carries the same BC type (one type per run isolates each flux)."""
    for dim in (2, 3):
        mesh = periodic_box(dim, 2, 3, 0.0, 1.0, affine=_affine(dim, 3), bcs=[0] * (2 * dim))
        base = cases.free_stream(mesh, rho=1.1, vel=[0.3, 0.2, -0.1][:dim], p=2.0)
        u = cases.perturbed(mesh, base, amp=0.2, seed=dim)
        bc = [make_golden.bc_example(kind, dim)]
        for q in (0, 1):
            ref = oracle_mod.Oracle(mesh, quirks=q, bcs=bc).rhs(u)
            op = _op(mesh, quirks=q and "fixed" or "reference", bcs=bc)
            d = np.empty_like(u)
            op.Mult(u, d)
            assert normalized_error(d, ref["dudt"], mesh.num_fields) <= RHS_TOL, (kind, dim, q)
            op.close()


def test_boundary_free_stream_preserved_gpu():
    """A uniform state is kept by inflow of that state, outflow, pressure
    outflow at its pressure, Riemann invariants of that state and subsonic
    inflow of its density and velocity; flow along x is kept between slip walls
    and between symmetry planes."""
    for dim in (2, 3):
        vel = [0.3, -0.2, 0.1][:dim]
        mesh = periodic_box(dim, 3, 3, 0.0, 1.0, bcs=list(range(2 * dim)))
        u = cases.free_stream(mesh, rho=1.2, vel=vel, p=2.0)
        state = list(u.reshape(dim + 2, -1)[:, 0])
        prim = [1.2] + vel + [2.0]
        for kind in ("state", "outflow", "pressure_outflow", "riemann", "inflow_rv"):
            data = {"state": state, "riemann": prim, "inflow_rv": prim[:-1]}.get(kind)
            bc = [(kind, data, 2.0 if kind == "pressure_outflow" else None)]
            op = _op(mesh, quirks="fixed", bcs=bc * (2 * dim))
            d = np.empty_like(u)
            op.Mult(u, d)
            assert np.abs(d).max() < 1e-12, (dim, kind)
            op.close()
    mesh = periodic_box(2, 3, 3, 0.0, 1.0, bcs=[0, 0, 1, 1])
    u = cases.free_stream(mesh, rho=1.2, vel=[0.4, 0.0], p=2.0)
    for wall in ("slip_wall", "symmetry"):
        op = _op(mesh, quirks="fixed", bcs=[("outflow",), (wall,)])
        d = np.empty_like(u)
        op.Mult(u, d)
        assert np.abs(d).max() < 1e-12, wall
        op.close()


@pytest.mark.parametrize("scheme", ["RK3SSP", "LSRK45"])
def test_boundary_trajectory_matches_oracle(oracle_mod, scheme):
    mesh = periodic_box(2, 6, 3, 0.0, 1.0, bcs=SIDES[2])
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3], p=1.5)
    u0 = cases.perturbed(mesh, base, amp=0.1, seed=5)
    orc = oracle_mod.Oracle(mesh, quirks=1, bcs=BCS[2])
    lam = orc.rhs(u0)["lambda_max"]
    dt = 0.3 * mesh.hmin / (lam * (mesh.order + 1) ** 2)
    ref = orc.step(u0, dt, scheme=0 if scheme == "RK3SSP" else 1, nsteps=10)
    op = _op(mesh, quirks="fixed", bcs=BCS[2])
    u = u0.copy()
    op.Step(u, dt, scheme=scheme, nsteps=10)
    assert normalized_error(u, ref, mesh.num_fields) <= TRAJ_TOL
    op.close()


def test_boundary_fp32_rhs():
    from test_gpu_fp32 import rel_l2
    for dim in (2, 3):
        mesh = periodic_box(dim, 3, 3, 0.0, 1.0, affine=_affine(dim, 2), bcs=SIDES[dim])
        base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5)
        u = cases.perturbed(mesh, base, amp=0.1, seed=9)
        d64, d32 = np.empty_like(u), np.empty_like(u)
        op = _op(mesh, quirks="fixed", bcs=BCS[dim])
        op.Mult(u, d64)
        op.close()
        op = _op(mesh, quirks="fixed", bcs=BCS[dim], precision="fp32")
        op.Mult(u, d32)
        op.close()
        assert max(rel_l2(d32, d64, mesh.num_fields)) <= 2e-3


def test_boundary_solves_in_a_batch():
    """Bounded and periodic solves of one class share a batch launch; each
    matches its one-operator run."""
    from prandtl_b200.batch import Batch
    from prandtl_b200.ensemble import fixed_dt
    runs = []
    for dim, sides, bl in ((2, SIDES[2], False), (2, None, False), (3, SIDES[3], True), (3, None, True)):
        mesh = periodic_box(dim, 3, 3, 0.0, 1.0, affine=_affine(dim, 4), bcs=sides)
        base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5)
        u0 = cases.perturbed(mesh, base, amp=0.2, seed=dim)
        kw = dict(quirks="fixed", blending=bl, bcs=BCS[dim] if sides else None)
        runs.append((mesh, u0, kw, fixed_dt(mesh, u0, 0.3)))
    b = Batch("fp64", "LSRK45", arena_bytes=1 << 28)
    ids = [b.add(mesh, u0, dt=dt, nsteps=4, **kw) for mesh, u0, kw, dt in runs]
    b.advance(4)
    for sid, (mesh, u0, kw, dt) in zip(ids, runs):
        op = _op(mesh, **kw)
        ref = u0.copy()
        op.Step(ref, dt, scheme="LSRK45", nsteps=4)
        op.close()
        assert normalized_error(b.read(sid), ref, mesh.num_fields) <= 1e-12, kw
    b.close()


NS = dict(parabolic=True, **make_golden.PHYS)


@pytest.mark.parametrize("kind", ["noslip_adiabatic", "noslip_isothermal", "outflow", "state", "pressure_outflow",
                                  "riemann", "inflow_rv"])
def test_each_boundary_type_alone_navier_stokes(oracle_mod, kind):
    """Navier-Stokes: BR1 boundary lifting and the viscous boundary flux of each
    type on its own, both quirk modes (Riemann invariants: fixed mode only)."""
    for dim in (2, 3):
        mesh = periodic_box(dim, 2, 3, 0.0, 1.0, affine=_affine(dim, 3), bcs=[0] * (2 * dim))
        base = cases.free_stream(mesh, rho=1.1, vel=[0.3, 0.2, -0.1][:dim], p=2.0)
        u = cases.perturbed(mesh, base, amp=0.2, seed=dim)
        bc = [make_golden.bc_example(kind, dim)]
        for q in ((1,) if kind == "riemann" else (0, 1)):
            ref = oracle_mod.Oracle(mesh, quirks=q, bcs=bc, **NS).rhs(u)
            op = _op(mesh, quirks=q and "fixed" or "reference", bcs=bc, **NS)
            d = np.empty_like(u)
            op.Mult(u, d)
            assert normalized_error(d, ref["dudt"], mesh.num_fields) <= RHS_TOL, (kind, dim, q)
            op.close()


def test_fluid_at_rest_between_no_slip_walls():
    """A uniform state at rest stays at rest between adiabatic walls (no heat
    flux) and isothermal walls at its own temperature.  (Reference mode in 3D
    is not free-stream preserving: its zeta-loop flux mix-up, Q2.)"""
    for dim in (2, 3):
        mesh = periodic_box(dim, 3, 3, 0.0, 1.0, affine=_affine(dim, 6), bcs=[0, 0] + [1] * (2 * dim - 2))
        u = cases.free_stream(mesh, rho=1.2, vel=[0.0] * dim, p=1.5)
        T = 1.5 / (1.2 * make_golden.PHYS["R_gas"])
        bcs = [("noslip_adiabatic", dict(wall_vel=[0.0] * dim, heat_flux=0.0)),
               ("noslip_isothermal", dict(wall_vel=[0.0] * dim, wall_T=T))]
        for quirks in (("reference", "fixed") if dim == 2 else ("fixed",)):
            op = _op(mesh, quirks=quirks, bcs=bcs, **NS)
            d = np.empty_like(u)
            op.Mult(u, d)
            assert np.abs(d).max() < 1e-12, (dim, quirks)
            op.close()


@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_lid_driven_cavity_trajectory_matches_oracle(oracle_mod, quirks):
    """2D lid-driven cavity (moving adiabatic lid, three adiabatic walls at
    rest), 10 LSRK4(5) steps against the oracle."""
    mesh = periodic_box(2, 4, 3, 0.0, 1.0, bcs=[1, 1, 1, 0])
    u0 = cases.free_stream(mesh, rho=1.0, vel=[0.0, 0.0], p=1.0 / 1.4 / 0.1 ** 2)
    bcs = [("noslip_adiabatic", dict(wall_vel=[1.0, 0.0], heat_flux=0.0)),
           ("noslip_adiabatic", dict(wall_vel=[0.0, 0.0], heat_flux=0.0))]
    kw = dict(mu=0.01, Pr=0.71, parabolic=1)
    q = 0 if quirks == "reference" else 1
    orc = oracle_mod.Oracle(mesh, quirks=q, bcs=bcs, **kw)
    lam = orc.rhs(u0)["lambda_max"]
    dt = 0.3 * mesh.hmin / ((lam + 1.0) * (mesh.order + 1) ** 2)
    ref = orc.step(u0, dt, scheme=1, nsteps=10)
    op = _op(mesh, quirks=quirks, bcs=bcs, mu=0.01, Pr=0.71, parabolic=True)
    u = u0.copy()
    op.Step(u, dt, scheme="LSRK45", nsteps=10)
    assert normalized_error(u - u0, ref - u0, mesh.num_fields) <= 1e-9
    assert np.abs(ref - u0).max() > 1e-6   # the lid has set the fluid moving
    op.close()


def test_navier_stokes_boundary_fp32_and_batch():
    """FP32-bulk form within 2e-3 relative L2 of FP64 for one RHS; bounded NS
    solves in a batch match their one-operator runs (FP64, 1e-12)."""
    from prandtl_b200.batch import Batch
    from prandtl_b200.ensemble import fixed_dt
    from test_gpu_fp32 import rel_l2
    runs = []
    for dim in (2, 3):
        mesh = periodic_box(dim, 3, 3, 0.0, 1.0, affine=_affine(dim, 2), bcs=make_golden.NS_WALL_SIDES[dim])
        base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5)
        u = cases.perturbed(mesh, base, amp=0.1, seed=9)
        for quirks in ("reference", "fixed"):
            kw = dict(quirks=quirks, bcs=make_golden.NS_BCS[dim], **NS)
            d64, d32 = np.empty_like(u), np.empty_like(u)
            op = _op(mesh, **kw)
            op.Mult(u, d64)
            op.close()
            op = _op(mesh, precision="fp32", **kw)
            op.Mult(u, d32)
            op.close()
            assert max(rel_l2(d32, d64, mesh.num_fields)) <= 2e-3, (dim, quirks)
            runs.append((mesh, u, kw, fixed_dt(mesh, u, 0.3)))
    b = Batch("fp64", "LSRK45", arena_bytes=1 << 28)
    ids = [b.add(mesh, u0, dt=dt, nsteps=3, **kw) for mesh, u0, kw, dt in runs]
    b.advance(3)
    for sid, (mesh, u0, kw, dt) in zip(ids, runs):
        op = _op(mesh, **kw)
        ref = u0.copy()
        op.Step(ref, dt, scheme="LSRK45", nsteps=3)
        op.close()
        assert normalized_error(b.read(sid), ref, mesh.num_fields) <= 1e-12, kw["quirks"]
    b.close()
