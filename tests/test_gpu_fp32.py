"""FP32-bulk form (precision="fp32") against the FP64 path (marked gpu).

The bulk two-point flux, surface flux and gradient work runs in FP32 while
primitives, the RK state and registers stay FP64.  Tolerances: one RHS
evaluation within 2e-3 relative L2 of the FP64 RHS (at Mach 0.1 the momentum
and energy rates are small differences of O(p) fluxes, so FP32 loses about
three digits there); after 50 LSRK4(5) steps the state within 1e-5 relative
L2 (density, momentum, energy), the target stated for this form.
"""
import numpy as np
import pytest

from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

pytestmark = pytest.mark.gpu


def _op(mesh, **kw):
    from prandtl_b200.operator import DGSEMOperator
    return DGSEMOperator(mesh, **kw)


def rel_l2(a, b, nf):
    """Relative L2 error of density, momentum (as one vector) and energy."""
    a, b = a.reshape(nf, -1), b.reshape(nf, -1)
    groups = [[0], list(range(1, nf - 1)), [nf - 1]]
    return [float(np.linalg.norm(a[g] - b[g]) / max(np.linalg.norm(b[g]), 1e-300)) for g in groups]


TGV = dict(parabolic=True, mu=1 / 1600, Pr=0.71, quirks="fixed")


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_fp32_rhs_tgv(order):
    mesh = periodic_box(3, 4 if order < 4 else 3, order, 0.0, 2 * np.pi)
    u = cases.taylor_green(mesh)
    d64, d32 = np.empty_like(u), np.empty_like(u)
    _op(mesh, **TGV).Mult(u, d64)
    op32 = _op(mesh, precision="fp32", **TGV)
    op32.Mult(u, d32)
    errs = rel_l2(d32, d64, mesh.num_fields)
    assert max(errs) <= 2e-3, errs


@pytest.mark.parametrize("dim,order", [(2, 3), (3, 3), (2, 4), (3, 4), (3, 5)])
def test_fp32_rhs_reference_mode_navier_stokes(dim, order):
    """Reference-mode NS (gradient form, the reference's defects kept) in FP32:
    line tasks up to N = 4 (3D: 32- and 64-lane groups, where the eta flux
    replaces a zeta line's lower partners) and the pair form at N = 5."""
    mesh = periodic_box(dim, 3, order, 0.0, 1.0, affine=np.eye(dim) + 0.1 * np.eye(dim, k=1))
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5)
    u = cases.perturbed(mesh, base, amp=0.1, seed=4)
    kw = dict(parabolic=True, mu=0.01, Pr=0.71, quirks="reference")
    d64, d32 = np.empty_like(u), np.empty_like(u)
    _op(mesh, **kw).Mult(u, d64)
    _op(mesh, precision="fp32", **kw).Mult(u, d32)
    assert max(rel_l2(d32, d64, mesh.num_fields)) <= 2e-3


def test_fp32_rhs_euler_blended():
    mesh = periodic_box(2, 16, 3, -1.0, 1.0)
    u = cases.kelvin_helmholtz(mesh)
    d64, d32 = np.empty_like(u), np.empty_like(u)
    op64 = _op(mesh, blending=True)
    op64.Mult(u, d64)
    op32 = _op(mesh, blending=True, precision="fp32")
    op32.Mult(u, d32)
    assert (op64.alpha() > 0).any()
    np.testing.assert_allclose(op32.alpha(), op64.alpha(), rtol=0, atol=1e-5)
    assert max(rel_l2(d32, d64, 4)) <= 2e-3


@pytest.mark.parametrize("order", [2, 3, 4, 5])
def test_fp32_rhs_navier_stokes_blended(order):
    """Navier-Stokes with blending on a perturbed box: the line-task volume
    terms (N <= 3 and N = 5) and the indicator's cross-warp reduction (N >= 4)
    against the FP64 path."""
    mesh = periodic_box(3, 3, order, 0.0, 1.0, affine=np.eye(3) + 0.1 * np.eye(3, k=1))
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2], p=1.5)
    u = cases.perturbed(mesh, base, amp=0.3, seed=order)
    kw = dict(parabolic=True, blending=True, mu=0.01, Pr=0.71, quirks="fixed")
    d64, d32 = np.empty_like(u), np.empty_like(u)
    op64 = _op(mesh, **kw)
    op64.Mult(u, d64)
    op32 = _op(mesh, precision="fp32", **kw)
    op32.Mult(u, d32)
    assert (op64.alpha() > 0).any()
    np.testing.assert_allclose(op32.alpha(), op64.alpha(), rtol=0, atol=1e-5)
    assert max(rel_l2(d32, d64, mesh.num_fields)) <= 2e-3


@pytest.mark.parametrize("case", ["tgv", "ivortex"])
def test_fp32_trajectory_error(case):
    if case == "tgv":
        mesh = periodic_box(3, 8, 3, 0.0, 2 * np.pi)
        u0 = cases.taylor_green(mesh)
        kw = TGV
    else:
        mesh = periodic_box(2, 16, 3, 0.0, 10.0)
        u0 = cases.isentropic_vortex(mesh)
        kw = dict(quirks="fixed")
    op64 = _op(mesh, **kw)
    d = np.empty_like(u0)
    op64.Mult(u0, d)
    dt = op64.cfl_dt(0.1 if case == "tgv" else 0.5)
    u64, u32 = u0.copy(), u0.copy()
    op64.Step(u64, dt, scheme="LSRK45", nsteps=50)
    _op(mesh, precision="fp32", **kw).Step(u32, dt, scheme="LSRK45", nsteps=50)
    errs = rel_l2(u32, u64, mesh.num_fields)
    # relative to the change of the state over the run as well
    chg = rel_l2(u64, u0, mesh.num_fields)
    assert max(errs) <= 1e-5, (errs, chg)
