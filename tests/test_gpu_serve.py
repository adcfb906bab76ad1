"""Serving loop (prandtl_serve_*) on the GPU (marked gpu).

Requests that arrive while others are resident join the running batch.  Each
result must equal the same solve run alone, bit for bit, and match the
one-operator FP64 path within 1e-12 (FP64 server).
"""
import time

import numpy as np
import pytest

from prandtl_b200.batch import Server
from prandtl_b200.ensemble import Member, fixed_dt

pytestmark = pytest.mark.gpu


def _norm_err(g, r, nf):
    g, r = g.reshape(nf, -1), r.reshape(nf, -1)
    fl = np.maximum(np.abs(r).max(axis=1, keepdims=True), 1e-300)
    return float((np.abs(g - r) / np.maximum(np.abs(r), fl)).max())


REQS = [Member("ivortex", 4, 3, nsteps=9), Member("tgv", 3, 2, 0.1, 1600.0, nsteps=6),
        Member("tgv", 2, 3, 0.2, 300.0, nsteps=11), Member("ivortex", 5, 4, nsteps=4),
        Member("tgv", 2, 2, 0.3, 3000.0, nsteps=8)]


def _prep(m):
    mesh = m.mesh()
    u0 = m.initial_state(mesh)
    return mesh, u0, fixed_dt(mesh, u0, 0.3)


def test_results_alone_and_in_mix_identical_and_match_plain():
    from prandtl_b200.operator import DGSEMOperator
    prepped = [_prep(m) for m in REQS]
    alone = []
    for m, (mesh, u0, dt) in zip(REQS, prepped):
        s = Server("fp64", steps_per_tick=2, arena_bytes=1 << 28)
        t = s.submit(mesh, u0, dt=dt, nsteps=m.nsteps, **m.physics())
        alone.append(s.wait(t, 60.0)[0])
        s.close()
    s = Server("fp64", steps_per_tick=2, arena_bytes=1 << 29)
    tickets = []
    for m, (mesh, u0, dt) in zip(REQS, prepped):
        tickets.append(s.submit(mesh, u0, dt=dt, nsteps=m.nsteps, **m.physics()))
        time.sleep(0.003)   # staggered arrivals: later requests join a running batch
    mixed = [s.wait(t, 60.0) for t in tickets]
    st = s.stats()
    s.close()
    assert st["completed"] == len(REQS) and st["rejected"] == 0
    for k, (m, (mesh, u0, dt)) in enumerate(zip(REQS, prepped)):
        assert np.array_equal(alone[k], mixed[k][0])
        assert mixed[k][1] > 0
        op = DGSEMOperator(mesh, **m.physics())
        ref = u0.copy()
        op.Step(ref, dt, scheme="LSRK45", nsteps=m.nsteps)
        op.close()
        assert _norm_err(mixed[k][0], ref, mesh.num_fields) <= 1e-12


def test_admission_waits_for_room():
    # an arena that holds one solve: the second waits until the first retires
    m = Member("tgv", 3, 3, 0.1, 1600.0, nsteps=5)
    mesh, u0, dt = _prep(m)
    from prandtl_b200.batch import Batch
    b = Batch("fp32")
    need = b.footprint(mesh, **m.physics())
    b.close()
    s = Server("fp32", steps_per_tick=1, arena_bytes=need + need // 2)
    t1 = s.submit(mesh, u0, dt=dt, nsteps=5, **m.physics())
    t2 = s.submit(mesh, u0, dt=dt, nsteps=5, **m.physics())
    r1, s1 = s.wait(t1, 60.0)
    r2, s2 = s.wait(t2, 60.0)
    assert np.array_equal(r1, r2)
    assert s2 > s1
    st = s.stats()
    s.close()
    assert st["completed"] == 2
    assert st["steps"] >= 10   # never both resident: at least 5 + 5 batch steps


def test_request_larger_than_arena_rejected():
    from prandtl_b200._lib import PRANDTL_ENOMEM, PrandtlError
    m = Member("tgv", 6, 3, nsteps=2)          # about 3.4 MB of arena
    mesh, u0, dt = _prep(m)
    s = Server("fp64", arena_bytes=1 << 20)
    with pytest.raises(PrandtlError) as ei:
        s.submit(mesh, u0, dt=dt, nsteps=2, **m.physics())
    assert ei.value.status == PRANDTL_ENOMEM
    s.close()
