"""Non-affine (multilinear) elements on the GPU: the FP64 kernels with the
transformation at every node, the scaled normal at every face node and the
line-integrated subcell metrics (DGSEMIntegrator.cpp:254-267, :1199-1304;
LiftingBR1.cpp:40-49, :184-186), against the oracle and the reference's own
outputs (marked gpu).

Tolerance: per-DOF normalised error (conftest.normalized_error) <= 1e-12 for
one RHS evaluation; <= 1e-10 after the stated RK steps.
"""
import os
import sys

import numpy as np
import pytest

from conftest import normalized_error
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
TRAJ_TOL = 1e-10
GOLDEN = np.load(os.path.join(HERE, "golden", "reference_rhs.npz"))


def _op(mesh, **kw):
    from prandtl_b200.operator import DGSEMOperator
    return DGSEMOperator(mesh, **kw)


def _mesh(dim, n, order, amp=0.06, bcs=None):
    return periodic_box(dim, n, order, 0.0, 1.0, bcs=bcs, warp=make_golden.warp_field(dim, amp))


def _state(mesh, seed=0, amp=0.1):
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][: mesh.dim], p=1.5)
    return cases.perturbed(mesh, base, amp=amp, seed=seed)


PHYS = [
    dict(parabolic=0, blending=0),
    dict(parabolic=0, blending=1),
    dict(parabolic=1, blending=0, mu=0.01, Pr=0.71),
    dict(parabolic=1, blending=1, mu=0.01, Pr=0.71),
]


@pytest.mark.parametrize("dim,n,order", [(2, 3, 1), (2, 3, 2), (2, 3, 3), (2, 2, 4), (2, 2, 5),
                                         (3, 3, 1), (3, 3, 2), (3, 2, 3), (3, 2, 4), (3, 2, 5)])
@pytest.mark.parametrize("phys", range(len(PHYS)))
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_curved_rhs_matches_oracle(oracle_mod, dim, n, order, phys, quirks):
    kw = PHYS[phys]
    mesh = _mesh(dim, n, order, amp=0.05 if n == 3 else 0.0)
    if n == 2:   # corners of a 2-element lattice sit where the periodic warp vanishes: use a skew one
        mesh = periodic_box(dim, n, order, 0.0, 1.0,
                            warp=lambda X: 0.04 * np.stack([np.sin(2 * np.pi * (X[(d + 1) % dim] + 0.13 * d + 0.1))
                                                            for d in range(dim)]))
    assert not mesh.affine
    u = _state(mesh, seed=order + 10 * dim, amp=0.3 if kw["blending"] else 0.1)
    q = 0 if quirks == "reference" else 1
    ref = oracle_mod.Oracle(mesh, quirks=q, **kw).rhs(u, want_alpha=True)
    op = _op(mesh, quirks=quirks, **kw)
    d = np.empty_like(u)
    op.Mult(u, d)
    err = normalized_error(d, ref["dudt"], mesh.num_fields)
    assert err <= RHS_TOL, f"normalised error {err:.3e}"
    assert abs(op.GetMaxCharSpeed() - ref["lambda_max"]) <= 1e-13 * ref["lambda_max"]
    if kw["blending"]:
        np.testing.assert_allclose(op.alpha(), ref["alpha"], rtol=0, atol=1e-12)
        assert (ref["alpha"] > 0).any()


@pytest.mark.parametrize("case", make_golden.CURVED_CASES, ids=[c[0] for c in make_golden.CURVED_CASES])
def test_curved_rhs_matches_reference_golden(case):
    """The reference's own outputs on multilinear elements (reference mode)."""
    name, dim, n, order, par, bl, amp, seed, bset = case
    mesh, u = make_golden.curved_inputs(dim, n, order, amp, seed, bset)
    np.testing.assert_array_equal(u, GOLDEN[f"{name}/u"])
    bcs = make_golden.BC_SETS[bset][1][dim] if bset else None
    op = _op(mesh, parabolic=bool(par), blending=bool(bl), quirks="reference", bcs=bcs, **make_golden.PHYS)
    d = np.empty_like(u)
    op.Mult(u, d)
    assert normalized_error(d, GOLDEN[f"{name}/dudt"], mesh.num_fields) <= RHS_TOL
    if bl:
        np.testing.assert_allclose(op.alpha(), GOLDEN[f"{name}/alpha"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("case", make_golden.CURVED_AXI_CASES, ids=[c[0] for c in make_golden.CURVED_AXI_CASES])
def test_curved_axisymmetric_matches_reference_golden(case):
    name, n, order, bl, amp, seed = case
    mesh, u = make_golden.curved_axi_inputs(n, order, bl, amp, seed)
    op = _op(mesh, blending=bool(bl), bcs=make_golden.AXI_BCS, axisymmetric=True)
    d = np.empty_like(u)
    op.Mult(u, d)
    assert normalized_error(d, GOLDEN[f"{name}/dudt"], mesh.num_fields) <= RHS_TOL


@pytest.mark.parametrize("kind", ["state", "outflow", "slip_wall", "symmetry", "riemann", "inflow_rv"])
def test_curved_boundaries_match_oracle(oracle_mod, kind):
    bcs = [make_golden.bc_example(kind, 2)]
    mesh = _mesh(2, 3, 3, bcs=[0, 0, 0, 0])
    u = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.1, vel=[0.35, -0.2], p=1.6), amp=0.2, seed=3)
    ref = oracle_mod.Oracle(mesh, quirks=0, blending=1, bcs=bcs).rhs(u)["dudt"]
    op = _op(mesh, blending=True, bcs=bcs)
    d = np.empty_like(u)
    op.Mult(u, d)
    assert normalized_error(d, ref, mesh.num_fields) <= RHS_TOL


@pytest.mark.parametrize("kind", ["noslip_adiabatic", "noslip_isothermal", "outflow"])
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_curved_ns_walls_match_oracle(oracle_mod, kind, quirks):
    bcs = [make_golden.bc_example(kind, 2)]
    mesh = _mesh(2, 3, 3, bcs=[0, 0, 0, 0])
    u = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.1, vel=[0.35, -0.2], p=1.6), amp=0.2, seed=4)
    q = 0 if quirks == "reference" else 1
    kw = dict(parabolic=1, blending=0, bcs=bcs, **make_golden.PHYS)
    ref = oracle_mod.Oracle(mesh, quirks=q, **kw).rhs(u)["dudt"]
    op = _op(mesh, quirks=quirks, **{**kw, "parabolic": True})
    d = np.empty_like(u)
    op.Mult(u, d)
    assert normalized_error(d, ref, mesh.num_fields) <= RHS_TOL


@pytest.mark.parametrize("scheme", ["RK3SSP", "LSRK45"])
@pytest.mark.parametrize("dim,order,par", [(2, 3, 0), (2, 2, 1), (3, 2, 1)])
def test_curved_trajectory_matches_oracle(oracle_mod, scheme, dim, order, par):
    mesh = _mesh(dim, 3, order)
    kw = dict(parabolic=par, blending=1 - par, mu=0.01, Pr=0.71)
    u0 = _state(mesh, seed=5, amp=0.2)
    orc = oracle_mod.Oracle(mesh, quirks=1, **kw)
    dt = 0.3 * mesh.hmin / (orc.rhs(u0)["lambda_max"] * (order + 1) ** 2)
    steps = 10
    ref = orc.step(u0, dt, scheme=0 if scheme == "RK3SSP" else 1, nsteps=steps)
    op = _op(mesh, quirks="fixed", **{**kw, "parabolic": bool(par), "blending": bool(1 - par)})
    u = u0.copy()
    op.Step(u, dt, scheme=scheme, nsteps=steps)
    assert normalized_error(u, ref, mesh.num_fields) <= TRAJ_TOL


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 3), (3, 2), (3, 3)])
def test_curved_free_stream_preserved(dim, order):
    """Uniform flow stays uniform on multilinear elements (metric identities of
    the nodal adjugates: 2D for N >= 1, 3D for N >= 2)."""
    mesh = _mesh(dim, 3, order)
    u = cases.free_stream(mesh, rho=1.2, vel=[0.3, -0.2, 0.1][:dim], p=1.5)
    for par in (False, True):
        op = _op(mesh, parabolic=par, quirks="fixed", mu=0.01)
        d = np.empty_like(u)
        op.Mult(u, d)
        assert np.abs(d).max() < 1e-12


def test_curved_conservation_budget():
    """Periodic warped mesh: the GPU budget sums with det J at every node give
    zero mass / momentum / energy rates to round-off."""
    mesh = _mesh(2, 4, 3)
    u = _state(mesh, seed=9, amp=0.2)
    op = _op(mesh, blending=True)
    d = np.empty_like(u)
    op.Mult(u, d)
    b = op.budgets(u, d)
    wJ = mesh.node_weights()
    host = (wJ[None, :] * d.reshape(4, -1)).sum(1)
    np.testing.assert_allclose(b["rates"][:4], host, rtol=0, atol=1e-12)
    assert np.abs(host).max() < 1e-12
    np.testing.assert_allclose(b["conserved"][0], (wJ * u.reshape(4, -1)[0]).sum(), rtol=1e-13)


def test_curved_rejected_where_not_built():
    """FP32-bulk Navier-Stokes handles and batches take affine meshes only."""
    from prandtl_b200 import _lib
    mesh = _mesh(2, 3, 2)
    with pytest.raises(_lib.PrandtlError) as ei:
        _op(mesh, precision="fp32", parabolic=True)
    assert ei.value.status == _lib.PRANDTL_EUNSUPPORTED
    from prandtl_b200.batch import Batch
    b = Batch(precision="fp64", arena_bytes=64 << 20)
    try:
        with pytest.raises(_lib.PrandtlError) as ei:
            b.add(mesh, cases.free_stream(mesh), dt=1e-3, nsteps=1)
        assert ei.value.status == _lib.PRANDTL_EUNSUPPORTED
    finally:
        b.close()


# ---------------------------------------------------------------- the axisymmetric ramp
@pytest.mark.parametrize("order,nx,ny", [(1, 20, 10), (2, 12, 6)])
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_ramp_rhs_matches_oracle(oracle_mod, order, nx, ny, quirks):
    """The reference's Ramp case (axisymmetric, blended, trapezoidal cells over
    the cone; inflow, outflow, axis and slip-wall boundaries) on a coarse mesh,
    from a perturbed Mach-2 state so the indicator fires."""
    mesh = cases.ramp_mesh(order, nx, ny)
    assert not mesh.affine
    U = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.0, vel=[2.0, 0.0], p=1 / 1.4),
                        amp=0.3, seed=order).reshape(4, -1)
    u = (U * mesh.coords[1][None, :]).reshape(-1)
    q = 0 if quirks == "reference" else 1
    ref = oracle_mod.Oracle(mesh, quirks=q, blending=1, bcs=cases.RAMP_BCS, axisymmetric=1).rhs(u, want_alpha=True)
    assert (ref["alpha"] > 0).any()
    op = _op(mesh, quirks=quirks, blending=True, bcs=cases.RAMP_BCS, axisymmetric=True)
    d = np.empty_like(u)
    op.Mult(u, d)
    assert normalized_error(d, ref["dudt"], 4) <= RHS_TOL
    np.testing.assert_allclose(op.alpha(), ref["alpha"], rtol=0, atol=1e-12)


def test_ramp_trajectory_matches_oracle(oracle_mod):
    """100 SSP-RK3 steps of the ramp flow from the reference's initial state:
    the shock forms off the cone and the blending follows it."""
    mesh = cases.ramp_mesh(1, 24, 12)
    u0 = cases.ramp_ic(mesh)
    orc = oracle_mod.Oracle(mesh, quirks=0, blending=1, bcs=cases.RAMP_BCS, axisymmetric=1)
    dt = 0.3 * mesh.hmin / (3.0 * 4)
    ref = orc.step(u0, dt, scheme=0, nsteps=100)
    op = _op(mesh, quirks="reference", blending=True, bcs=cases.RAMP_BCS, axisymmetric=True)
    u = u0.copy()
    op.Step(u, dt, scheme="RK3SSP", nsteps=100)
    assert normalized_error(u, ref, 4) <= TRAJ_TOL
    assert (orc.rhs(ref, want_alpha=True)["alpha"] > 0).any()


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 3), (3, 2)])
def test_curved_fp32_euler_tracks_fp64(dim, order):
    """The FP32-bulk Euler form on multilinear elements: the same state after
    20 LSRK steps as the FP64 form within 1e-5 relative L2 per field (the
    FP32-bulk tolerance), with blending."""
    mesh = _mesh(dim, 3, order)
    u0 = _state(mesh, seed=11, amp=0.2)
    dt = 0.2 * mesh.hmin / (2.0 * (order + 1) ** 2)
    u64, u32 = u0.copy(), u0.copy()
    _op(mesh, blending=True, quirks="fixed").Step(u64, dt, scheme="LSRK45", nsteps=20)
    _op(mesh, blending=True, quirks="fixed", precision="fp32").Step(u32, dt, scheme="LSRK45", nsteps=20)
    a, b = u32.reshape(mesh.num_fields, -1), u64.reshape(mesh.num_fields, -1)
    for f in range(mesh.num_fields):
        assert np.linalg.norm(a[f] - b[f]) <= 1e-5 * np.linalg.norm(b[f])
    assert not np.array_equal(a, b)   # the FP32 kernels did run


def test_ramp_fp32_tracks_fp64():
    """The Ramp case in the FP32-bulk form (axisymmetric, blended, multilinear)
    against the FP64 form after 200 SSP-RK3 steps at the reference's dt."""
    mesh = cases.ramp_mesh(1, 24, 12)
    u0 = cases.ramp_ic(mesh)
    kw = dict(quirks="reference", blending=True, bcs=cases.RAMP_BCS, axisymmetric=True)
    u64, u32 = u0.copy(), u0.copy()
    _op(mesh, **kw).Step(u64, 1e-3, scheme="RK3SSP", nsteps=200)
    _op(mesh, precision="fp32", **kw).Step(u32, 1e-3, scheme="RK3SSP", nsteps=200)
    a, b = u32.reshape(4, -1), u64.reshape(4, -1)
    for f in range(4):
        assert np.linalg.norm(a[f] - b[f]) <= 1e-5 * np.linalg.norm(b[f])
