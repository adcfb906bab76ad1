"""FP64 device budgets (prandtl_budgets, marked gpu): integrals of the
conserved fields and of the entropy function, their rates and the entropy
production, against the same sums formed on the host; conservation and entropy
conservation read through them; FP32-bulk runs keep mass and energy."""
import numpy as np
import pytest

from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

pytestmark = pytest.mark.gpu


def _op(mesh, **kw):
    from prandtl_b200.operator import DGSEMOperator
    return DGSEMOperator(mesh, **kw)


def host_budgets(mesh, u, dudt, gamma=1.4):
    nf, dim = mesh.num_fields, mesh.dim
    U, wJ = u.reshape(nf, -1), mesh.node_weights()
    rho, vel = U[0], U[1:1 + dim] / U[0]
    vv = np.sum(vel ** 2, 0)
    p = (gamma - 1) * (U[-1] - 0.5 * rho * vv)
    s = np.log(p) - gamma * np.log(rho)
    beta = rho / p
    v = np.concatenate([((gamma - s) / (gamma - 1) - 0.5 * beta * vv)[None], beta * vel, -beta[None]])
    D = dudt.reshape(nf, -1)
    return {"conserved": (wJ * U).sum(1), "entropy": float(np.sum(wJ * (-rho * s / (gamma - 1)))),
            "rates": (wJ * D).sum(1), "entropy_rate": float(np.sum(wJ * np.sum(v * D, 0))),
            "scale": float(np.sum(wJ * np.sum(np.abs(v * D), 0)))}


@pytest.mark.parametrize("dim,order", [(2, 3), (3, 2), (3, 4)])
def test_budgets_match_host_sums(dim, order):
    mesh = periodic_box(dim, 3, order, 0.0, 1.0, affine=np.eye(dim) + 0.1 * np.eye(dim, k=1))
    u = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5), amp=0.2, seed=3)
    op = _op(mesh, quirks="fixed", parabolic=True, mu=0.01, Pr=0.71)
    d = np.empty_like(u)
    op.Mult(u, d)
    g, h = op.budgets(u, d), host_budgets(mesh, u, d)
    np.testing.assert_allclose(g["conserved"], h["conserved"], rtol=1e-13)
    assert abs(g["entropy"] - h["entropy"]) <= 1e-13 * abs(h["entropy"])
    scale = np.abs(h["rates"]).max() + np.abs(h["conserved"]).max()
    np.testing.assert_allclose(g["rates"], h["rates"], rtol=0, atol=1e-13 * scale)
    assert abs(g["entropy_rate"] - h["entropy_rate"]) <= 1e-13 * h["scale"]
    g2 = op.budgets(u)
    assert (g2["rates"] == 0).all() and g2["entropy_rate"] == 0 and (g2["conserved"] == g["conserved"]).all()
    import torch
    gd = op.budgets(torch.from_numpy(u).cuda(), torch.from_numpy(d).cuda())
    assert (gd["conserved"] == g["conserved"]).all() and gd["entropy_rate"] == g["entropy_rate"]
    op.close()


def test_budgets_read_conservation_and_entropy_conservation():
    """Periodic, fixed mode, entropy-conservative surface flux, no viscosity:
    every conserved rate and the entropy production vanish to round-off."""
    for dim in (2, 3):
        mesh = periodic_box(dim, 4, 3, 0.0, 1.0, affine=np.eye(dim) + 0.1 * np.eye(dim, k=1))
        u = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][:dim], p=1.5),
                            amp=0.2, seed=4)
        op = _op(mesh, quirks="fixed", surface_dissipation=False)
        d = np.empty_like(u)
        op.Mult(u, d)
        g, h = op.budgets(u, d), host_budgets(mesh, u, d)
        assert abs(g["entropy_rate"]) <= 1e-13 * h["scale"]
        wabs = (mesh.node_weights() * np.abs(d.reshape(mesh.num_fields, -1))).sum(1)
        assert (np.abs(g["rates"]) <= 1e-13 * wabs).all()
        op.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_budgets_over_a_trajectory(precision):
    """TGV, 20 LSRK4(5) steps: mass and energy change by round-off only (FP64
    RK state in both forms); the entropy function decreases."""
    mesh = periodic_box(3, 4, 3, 0.0, 2 * np.pi)
    u0 = cases.taylor_green(mesh)
    op = _op(mesh, parabolic=True, mu=1 / 1600, Pr=0.71, quirks="fixed", precision=precision)
    d = np.empty_like(u0)
    op.Mult(u0, d)
    b0 = op.budgets(u0)
    u = u0.copy()
    op.Step(u, op.cfl_dt(0.2, op.GetMaxCharSpeed()), scheme="LSRK45", nsteps=20)
    b1 = op.budgets(u)
    # measured: FP64 0 and 1.6e-16, FP32-bulk 5.4e-11 and 5.6e-11 (mass, energy);
    # entropy -2.34e-8 in both forms
    tol = 1e-13 if precision == "fp64" else 1e-9
    drift = [abs(b1["conserved"][f] - b0["conserved"][f]) / abs(b0["conserved"][f]) for f in (0, 4)]
    dS = (b1["entropy"] - b0["entropy"]) / abs(b0["entropy"])
    assert max(drift) <= tol, drift
    assert -1e-6 <= dS <= 0.0, dS
    op.close()


def test_batch_budgets_match_the_operator():
    """A batch solve's budgets read in place equal the operator's on the same
    state, before and after steps (FP32-bulk batch: mass and energy kept)."""
    from prandtl_b200.batch import Batch
    mesh = periodic_box(3, 3, 3, 0.0, 2 * np.pi)
    u0 = cases.taylor_green(mesh, mach=0.2)
    phys = dict(parabolic=True, mu=1 / 400, Pr=0.71, quirks="fixed")
    b = Batch("fp32", "LSRK45", arena_bytes=1 << 28)
    sid = b.add(mesh, u0, dt=2e-3, nsteps=10, **phys)
    op = _op(mesh, **phys)
    b0 = b.budgets(sid)
    r0 = op.budgets(u0)
    np.testing.assert_array_equal(b0["conserved"], r0["conserved"])
    assert b0["entropy"] == r0["entropy"]
    b.advance(10)
    b1 = b.budgets(sid)
    r1 = op.budgets(b.read(sid))
    np.testing.assert_array_equal(b1["conserved"], r1["conserved"])
    for f in (0, 4):
        assert abs(b1["conserved"][f] - b0["conserved"][f]) <= 1e-9 * abs(b0["conserved"][f])
    assert b1["entropy"] <= b0["entropy"]
    op.close()
    b.close()
