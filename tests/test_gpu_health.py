"""State checks and bounded waits (marked gpu).

The reference aborts when rho turns NaN (Simulation.cpp:1024-1035, every
nancheck_steps steps).  Here every RK stage checks every node of the state
it writes: a non-finite value, density <= 0 or pressure <= 0 sets a sticky
flag (PRANDTL_HEALTH_*), reported as PRANDTL_ENONFINITE by the one-operator
step (host pointers) or the next synchronize (device pointers), and per solve
by a batch (the failing solve alone stops; the others go on) and the serving
loop (that request alone fails).  Failures are injected on the host, in the
initial state; no GPU fault is involved.
"""
import time

import numpy as np
import pytest

from prandtl_b200 import _lib, cases
from prandtl_b200.batch import Batch, Server
from prandtl_b200.ensemble import Member, fixed_dt
from prandtl_b200.mesh import periodic_box
from prandtl_b200.operator import DGSEMOperator

pytestmark = pytest.mark.gpu

NS = dict(parabolic=True, mu=1.0 / 400.0, Pr=0.71, quirks="fixed")


def _tgv(n=3, order=3):
    mesh = periodic_box(3, n, order, 0.0, 2 * np.pi)
    u = cases.taylor_green(mesh)
    return mesh, u, fixed_dt(mesh, u, 0.2)


def _poison(mesh, u, how):
    v = u.reshape(mesh.num_fields, -1).copy()
    q = mesh.ndof // 2
    if how == "nan":
        v[2, q] = np.nan
    elif how == "density":
        v[0, q] = -0.5
    elif how == "pressure":   # energy below the kinetic energy: p < 0
        v[-1, q] = 0.0
    return v.reshape(-1)


@pytest.mark.parametrize("how", ["nan", "density", "pressure"])
@pytest.mark.parametrize("scheme", ["LSRK45", "RK3SSP"])
def test_step_reports_enonfinite(how, scheme):
    """A NaN, a negative density or an energy below the kinetic energy in the
    initial state: the logarithmic means of the two-point fluxes turn the
    element's RHS non-finite within the first stage, so the check reports
    non-finite values."""
    mesh, u, dt = _tgv()
    op = DGSEMOperator(mesh, **NS)
    bad = _poison(mesh, u, how)
    with pytest.raises(_lib.PrandtlError) as ei:
        op.Step(bad, dt, scheme=scheme, nsteps=2)
    assert ei.value.status == _lib.PRANDTL_ENONFINITE
    assert "admissible set" in str(ei.value)
    # reporting cleared the flag: a healthy state steps cleanly afterwards
    good = u.copy()
    op.Step(good, dt, scheme=scheme, nsteps=2)
    assert np.isfinite(good).all()
    op.close()


@pytest.mark.parametrize("scheme", ["LSRK45", "RK3SSP"])
def test_step_reports_positivity_loss(scheme):
    """A finite state whose first stage update drives density or pressure
    negative (a time step far beyond the CFL limit): the check names the
    positivity loss."""
    mesh, u, dt = _tgv()
    op = DGSEMOperator(mesh, **NS)
    v = u.copy()
    with pytest.raises(_lib.PrandtlError) as ei:
        op.Step(v, 2000.0 * dt, scheme=scheme, nsteps=1)
    assert ei.value.status == _lib.PRANDTL_ENONFINITE
    assert "density <= 0" in str(ei.value) or "pressure <= 0" in str(ei.value)
    op.close()


def test_device_pointer_step_reports_at_synchronize():
    torch = pytest.importorskip("torch")
    mesh, u, dt = _tgv()
    op = DGSEMOperator(mesh, **NS)
    ut = torch.from_numpy(_poison(mesh, u, "nan")).cuda()
    op.Step(ut, dt, scheme="LSRK45", nsteps=1)      # enqueued, no wait
    with pytest.raises(_lib.PrandtlError) as ei:
        op.synchronize()
    assert ei.value.status == _lib.PRANDTL_ENONFINITE
    op.synchronize()                                 # reported once, then clear
    op.close()


def test_healthy_trajectory_is_unchanged_by_the_check(oracle_mod):
    """The check only reads: a healthy LSRK trajectory still matches the oracle."""
    mesh, u, dt = _tgv(2, 3)
    op = DGSEMOperator(mesh, **NS)
    g = u.copy()
    op.Step(g, dt, scheme="LSRK45", nsteps=3)
    r = oracle_mod.Oracle(mesh, parabolic=1, mu=1.0 / 400.0, Pr=0.71, quirks=1).step(u, dt, scheme=1, nsteps=3)
    from conftest import normalized_error
    assert normalized_error(g, r, mesh.num_fields) <= 1e-10
    op.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_stops_only_the_failing_solve(precision):
    members = [Member("tgv", 2, 3, 0.1, 800.0), Member("tgv", 3, 2, 0.2, 400.0)]
    items = []
    for m in members:
        mesh = m.mesh()
        u0 = m.initial_state(mesh)
        items.append((m, mesh, u0, fixed_dt(mesh, u0, 0.2)))
    nsteps = 6
    # reference: the healthy member alone
    m1, mesh1, u1, dt1 = items[1]
    b0 = Batch(precision, "LSRK45", arena_bytes=1 << 28)
    s0 = b0.add(mesh1, u1, dt=dt1, nsteps=nsteps, **m1.physics())
    b0.advance(nsteps)
    alone = b0.read(s0)
    b0.close()

    b = Batch(precision, "LSRK45", arena_bytes=1 << 28)
    m0, mesh0, u0, dt0 = items[0]
    bad = b.add(mesh0, _poison(mesh0, u0, "density"), dt=dt0, nsteps=nsteps, **m0.physics())
    good = b.add(mesh1, u1, dt=dt1, nsteps=nsteps, **m1.physics())
    b.advance(nsteps)
    assert sorted(b.finished()) == sorted([bad, good])
    with pytest.raises(_lib.PrandtlError) as ei:
        b.query(bad)
    assert ei.value.status == _lib.PRANDTL_ENONFINITE
    assert "admissible set" in str(ei.value)
    with pytest.raises(_lib.PrandtlError):
        b.read(bad)
    q = b.query(good)
    assert q["steps_done"] == nsteps
    np.testing.assert_array_equal(b.read(good), alone)   # bit-identical alone and beside a failing solve
    b.close()


def test_server_fails_only_the_failing_request():
    mesh, u, dt = _tgv(2, 2)
    phys = dict(parabolic=True, mu=1.0 / 400.0, Pr=0.71, quirks="fixed")
    s = Server("fp64", steps_per_tick=2)
    t_ok1 = s.submit(mesh, u, dt=dt, nsteps=5, **phys)
    t_bad = s.submit(mesh, _poison(mesh, u, "nan"), dt=dt, nsteps=5, **phys)
    t_ok2 = s.submit(mesh, u, dt=dt, nsteps=5, **phys)
    r1, _ = s.wait(t_ok1, 120.0)
    with pytest.raises(_lib.PrandtlError) as ei:
        s.wait(t_bad, 120.0)
    assert ei.value.status == _lib.PRANDTL_ENONFINITE
    r2, _ = s.wait(t_ok2, 120.0)
    np.testing.assert_array_equal(r1, r2)
    assert np.isfinite(r1).all()
    # the server keeps serving after the failure
    t3 = s.submit(mesh, u, dt=dt, nsteps=5, **phys)
    r3, _ = s.wait(t3, 120.0)
    np.testing.assert_array_equal(r1, r3)
    s.close()


def test_batch_wait_times_out_then_recovers():
    """A host wait shorter than the enqueued work returns PRANDTL_ETIMEDOUT;
    the work itself is untouched and a later wait succeeds."""
    torch = pytest.importorskip("torch")
    m = Member("tgv", 12, 4, 0.1, 800.0)
    mesh = m.mesh()
    u0 = m.initial_state(mesh)
    b = Batch("fp64", "LSRK45", arena_bytes=1 << 30, timeout_s=2e-3, use_graph=False)
    sid = b.add(mesh, u0, dt=fixed_dt(mesh, u0, 0.1), nsteps=40, **m.physics())
    b.advance(40)
    with pytest.raises(_lib.PrandtlError) as ei:
        b.sync()
    assert ei.value.status == _lib.PRANDTL_ETIMEDOUT
    torch.cuda.synchronize()     # the device finishes the enqueued steps
    time.sleep(0.01)
    b.sync()
    assert b.query(sid)["steps_done"] == 40
    b.close()
