"""Axisymmetric (z, r) Euler on the GPU (marked gpu): the reference built with
AXISYMMETRIC, where the RK state is r U, the fluxes and boundary fluxes carry
r, the radial momentum gets + p, and the axis nodes keep a zero radial-momentum
rate (DGSEMOperator.cpp:161-533, DGSEMIntegrator.cpp, BdrFaceIntegrator.cpp).

Tolerances as for the planar parity tests: normalised per-DOF error <= 1e-12
for one RHS in FP64 (against the reference's own outputs and the oracle),
<= 1e-10 for trajectories; FP32 bulk within 2e-3 relative L2 of FP64.
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

BCS = make_golden.AXI_BCS


def _op(mesh, **kw):
    from prandtl_b200.operator import DGSEMOperator
    return DGSEMOperator(mesh, axisymmetric=True, **kw)


def test_axisymmetric_rhs_matches_reference_golden():
    gold = np.load(os.path.join(HERE, "golden", "reference_rhs.npz"))
    for name, n, order, bl, amp, seed in make_golden.AXI_CASES:
        mesh, u = make_golden.axi_inputs(n, order, bl, amp, seed)
        op = _op(mesh, blending=bool(bl), quirks="reference", bcs=BCS)
        d = np.empty_like(u)
        op.Mult(u, d)
        err = normalized_error(d, gold[f"{name}/dudt"], 4)
        assert err <= RHS_TOL, f"{name}: {err:.3e}"
        np.testing.assert_allclose(op.alpha(), gold[f"{name}/alpha"], rtol=0, atol=1e-12)
        op.close()


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("blending", [0, 1])
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_axisymmetric_rhs_matches_oracle(oracle_mod, order, blending, quirks):
    mesh, u = make_golden.axi_inputs((4, 3), order, blending, 0.3 if blending else 0.1, 40 + order)
    q = 0 if quirks == "reference" else 1
    ref = oracle_mod.Oracle(mesh, quirks=q, blending=blending, bcs=BCS, axisymmetric=1).rhs(u, want_alpha=True)
    op = _op(mesh, quirks=quirks, blending=bool(blending), bcs=BCS)
    d = np.empty_like(u)
    op.Mult(u, d)
    err = normalized_error(d, ref["dudt"], 4)
    assert err <= RHS_TOL, f"normalised error {err:.3e}"
    assert abs(op.GetMaxCharSpeed() - ref["lambda_max"]) <= 1e-13 * ref["lambda_max"]
    if blending:
        np.testing.assert_allclose(op.alpha(), ref["alpha"], rtol=0, atol=1e-12)
    axis = np.abs(mesh.coords[1]) <= 1e-14
    assert axis.any() and (d.reshape(4, -1)[2, axis] == 0).all()
    op.close()


@pytest.mark.parametrize("scheme", ["RK3SSP", "LSRK45"])
def test_axisymmetric_trajectory_matches_oracle(oracle_mod, scheme):
    mesh, u0 = make_golden.axi_inputs((6, 4), 3, 1, 0.2, 51)
    orc = oracle_mod.Oracle(mesh, quirks=0, blending=1, bcs=BCS, axisymmetric=1)
    lam = orc.rhs(u0)["lambda_max"]
    dt = 0.3 * mesh.hmin / (lam * (mesh.order + 1) ** 2)
    ref = orc.step(u0, dt, scheme=0 if scheme == "RK3SSP" else 1, nsteps=10)
    op = _op(mesh, quirks="reference", blending=True, bcs=BCS)
    u = u0.copy()
    op.Step(u, dt, scheme=scheme, nsteps=10)
    assert normalized_error(u, ref, 4) <= TRAJ_TOL
    op.close()


def test_axisymmetric_free_stream_preserved():
    """Uniform axial flow between the axis and a slip wall: the r-weighted
    pressure flux balances the source, in FP64 and the FP32-bulk form."""
    for N in (1, 2, 3, 4, 5):
        mesh = periodic_box(2, (4, 3), N, (0.0, 0.0), (2.0, 1.0), bcs=[0, 0, 1, 2])
        U = cases.free_stream(mesh, rho=1.2, vel=[0.3, 0.0], p=1.5).reshape(4, -1)
        rU = (U * mesh.coords[1][None, :]).reshape(-1)
        for prec, tol in (("fp64", 1e-12), ("fp32", 1e-4)):
            op = _op(mesh, quirks="fixed", bcs=[("outflow",), ("axis",), ("slip_wall",)], precision=prec)
            d = np.empty_like(rU)
            op.Mult(rU, d)
            assert np.abs(d).max() < tol, (N, prec, np.abs(d).max())
            op.close()


def test_axisymmetric_fp32_rhs():
    from test_gpu_fp32 import rel_l2
    mesh, u = make_golden.axi_inputs((5, 4), 3, 0, 0.1, 61)
    d64, d32 = np.empty_like(u), np.empty_like(u)
    op = _op(mesh, quirks="fixed", bcs=BCS)
    op.Mult(u, d64)
    op.close()
    op = _op(mesh, quirks="fixed", bcs=BCS, precision="fp32")
    op.Mult(u, d32)
    op.close()
    assert max(rel_l2(d32, d64, 4)) <= 2e-3


def test_axisymmetric_density_floor_matches_oracle(oracle_mod):
    """A raised axis density floor (the reference driver's 1e-8 rho_inf rule,
    here far above the density) sends every axis node to the nearest-node copy."""
    mesh, u = make_golden.axi_inputs((4, 3), 3, 1, 0.3, 71)
    for floor in (0.0, 100.0):
        ref = oracle_mod.Oracle(mesh, quirks=0, blending=1, bcs=BCS, axisymmetric=1,
                                axis_rho_floor=floor).rhs(u)["dudt"]
        op = _op(mesh, quirks="reference", blending=True, bcs=BCS, axis_rho_floor=floor)
        d = np.empty_like(u)
        op.Mult(u, d)
        assert normalized_error(d, ref, 4) <= RHS_TOL, floor
        op.close()


def test_recover_state_matches_oracle(oracle_mod):
    """The U behind the reference's axisymmetric output fields, host and device
    pointers; a planar operator refuses."""
    import ctypes as C
    import torch
    from prandtl_b200 import _lib
    mesh, u = make_golden.axi_inputs((4, 3), 4, 1, 0.3, 81)
    orc = oracle_mod.Oracle(mesh, quirks=0, bcs=BCS, axisymmetric=1)
    ref = np.empty_like(u)
    dp = C.POINTER(C.c_double)
    assert oracle_mod.lib().oracle_recover_weighted(C.byref(orc.m), C.byref(orc.c), u.ctypes.data_as(dp),
                                                    ref.ctypes.data_as(dp)) == 0
    op = _op(mesh, quirks="reference", bcs=BCS)
    np.testing.assert_array_equal(op.recover_state(u), ref)
    ud = torch.from_numpy(u).cuda()
    np.testing.assert_array_equal(op.recover_state(ud).cpu().numpy(), ref)
    op.close()
    from prandtl_b200.operator import DGSEMOperator
    planar = DGSEMOperator(periodic_box(2, 2, 2))
    with pytest.raises(_lib.PrandtlError):
        planar.recover_state(np.zeros(4 * planar.mesh.ndof))
    planar.close()
