"""Batched form (prandtl_batch_*) against the one-operator path (marked gpu).

A batch evaluates the same element arithmetic as the one-operator kernels,
through a persistent launch over many solves.  Each solve's state after k
steps must match the same solve stepped alone through DGSEMOperator.Step:
FP64 within 1e-12 (normalized per DOF), FP32 bulk within 1e-5 (FP32 rounding).  Results are
bit-identical whether a solve runs alone or among others, whether the steps
come from graph replays or direct launches, and before and after autotuning.
"""
import numpy as np
import pytest

from prandtl_b200 import cases
from prandtl_b200.batch import Batch
from prandtl_b200.ensemble import Member, fixed_dt, tgv_ensemble
from prandtl_b200.mesh import periodic_box

pytestmark = pytest.mark.gpu


def norm_err(g, r, nf):
    g, r = g.reshape(nf, -1), r.reshape(nf, -1)
    fl = np.maximum(np.abs(r).max(axis=1, keepdims=True), 1e-300)
    return float((np.abs(g - r) / np.maximum(np.abs(r), fl)).max())


def plain(member, u0, dt, nsteps, scheme="LSRK45", precision="fp64"):
    from prandtl_b200.operator import DGSEMOperator
    mesh = member.mesh()
    op = DGSEMOperator(mesh, precision=precision, **member.physics())
    u = u0.copy()
    op.Step(u, dt, scheme=scheme, nsteps=nsteps)
    op.close()
    return u


MIX = [Member("tgv", 3, 3, 0.1, 1600.0), Member("tgv", 2, 2, 0.2, 400.0), Member("tgv", 2, 5, 0.05, 3000.0),
       Member("ivortex", 4, 3), Member("tgv", 3, 1, 0.3, 100.0), Member("ivortex", 3, 4),
       Member("tgv", 2, 4, 0.15, 800.0)]


def _setup(members, cfl=0.3):
    out = []
    for m in members:
        mesh = m.mesh()
        u0 = m.initial_state(mesh)
        out.append((m, mesh, u0, fixed_dt(mesh, u0, cfl)))
    return out


@pytest.mark.parametrize("scheme", ["LSRK45", "RK3SSP"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_matches_plain(scheme, precision):
    items = _setup(MIX)
    nsteps = 7
    b = Batch(precision, scheme, arena_bytes=1 << 30, steps_per_graph=3)
    ids = [b.add(mesh, u0, dt=dt, nsteps=nsteps, **m.physics()) for m, mesh, u0, dt in items]
    b.advance(nsteps + 2)          # extra steps: every solve stops at its own count
    assert sorted(b.finished()) == sorted(ids)
    # FP32: the batch and one-shot kernels are compiled separately and may round
    # differently at contraction points; over 7 steps that stays below 1e-5
    # (normalized per DOF; the floor of the small w-momentum field is small)
    tol = 1e-12 if precision == "fp64" else 1e-5
    for sid, (m, mesh, u0, dt) in zip(ids, items):
        got = b.read(sid)
        ref = plain(m, u0, dt, nsteps, scheme, precision)
        assert norm_err(got, ref, mesh.num_fields) <= tol, (m, norm_err(got, ref, mesh.num_fields))
        q = b.query(sid)
        assert q["steps_left"] == 0 and q["steps_done"] == nsteps
    b.close()


def test_alone_and_in_mix_identical():
    items = _setup(MIX)
    target = 2
    m, mesh, u0, dt = items[target]
    alone = Batch("fp32", arena_bytes=1 << 28)
    a = alone.add(mesh, u0, dt=dt, nsteps=5, **m.physics())
    alone.advance(5)
    ua = alone.read(a)
    mix = Batch("fp32", arena_bytes=1 << 30)
    ids = [mix.add(mm, uu, dt=d, nsteps=5 if k == target else 3 + k, **x.physics())
           for k, (x, mm, uu, d) in enumerate(items)]
    mix.advance(12)
    um = mix.read(ids[target])
    assert np.array_equal(ua, um)


def test_graph_and_direct_launch_identical_and_admission_midway():
    items = _setup(MIX[:4])
    res = []
    for use_graph in (True, False):
        b = Batch("fp64", arena_bytes=1 << 30, use_graph=use_graph, steps_per_graph=2)
        first = [b.add(mesh, u0, dt=dt, nsteps=6, **m.physics()) for m, mesh, u0, dt in items[:2]]
        b.advance(3)
        late = [b.add(mesh, u0, dt=dt, nsteps=4, **m.physics()) for m, mesh, u0, dt in items[2:]]
        b.advance(5)
        res.append([b.read(i) for i in first + late])
        b.close()
    for x, y in zip(*res):
        assert np.array_equal(x, y)
    # the late arrivals took exactly their own 4 steps
    for k, (m, mesh, u0, dt) in enumerate(items[2:]):
        ref = plain(m, u0, dt, 4)
        assert norm_err(res[0][2 + k], ref, mesh.num_fields) <= 1e-12


def test_remove_and_reuse_arena_room():
    m = Member("tgv", 3, 3, 0.1, 1600.0)
    mesh = m.mesh()
    u0 = m.initial_state(mesh)
    dt = fixed_dt(mesh, u0, 0.3)
    b = Batch("fp64", max_solves=4)
    need = b.footprint(mesh, **m.physics())
    b.close()
    b = Batch("fp64", arena_bytes=2 * need + 4096, max_solves=4)
    x = b.add(mesh, u0, dt=dt, nsteps=2, **m.physics())
    y = b.add(mesh, u0, dt=dt, nsteps=2, **m.physics())
    from prandtl_b200._lib import PRANDTL_ENOMEM, PrandtlError
    with pytest.raises(PrandtlError) as ei:
        b.add(mesh, u0, dt=dt, nsteps=2, **m.physics())
    assert ei.value.status == PRANDTL_ENOMEM
    b.advance(2)
    ux = b.read(x)
    b.remove(x)
    z = b.add(mesh, ux, dt=dt, nsteps=2, **m.physics())   # continue x in y's neighbour slot
    b.advance(2)
    ref = plain(m, u0, dt, 4)
    assert norm_err(b.read(z), ref, mesh.num_fields) <= 1e-12
    assert np.array_equal(b.read(y), plain(m, u0, dt, 2)) or norm_err(b.read(y), plain(m, u0, dt, 2), 5) <= 1e-12
    b.close()


def test_autotuner_picks_a_timed_shape_and_keeps_results():
    items = _setup(MIX)
    b = Batch("fp32", arena_bytes=1 << 30)
    ids = [b.add(mesh, u0, dt=dt, nsteps=3, **m.physics()) for m, mesh, u0, dt in items]
    b.tune(reps=2)
    for m, mesh, _, _ in items:
        v, ms, lift_ms = b.class_info(mesh.dim, mesh.order, m.kind == "tgv")
        assert ms[v] > 0 and ms[v] == min(t for t in ms if t > 0)
        assert (lift_ms > 0) == (m.kind == "tgv")
    b.advance(3)
    for sid, (m, mesh, u0, dt) in zip(ids, items):
        ref = plain(m, u0, dt, 3, precision="fp32")
        assert norm_err(b.read(sid), ref, mesh.num_fields) <= 1e-5
    b.close()


def test_tuning_inside_steps_keeps_results():
    """The tuner inside the steps: the first n_variants steps of the advance
    time one launch shape each; the chosen shape is the fastest timed one and
    every solve's state equals the untuned batch's, bit for bit."""
    items = _setup(MIX)
    states = []
    for tuned in (False, True):
        b = Batch("fp32", arena_bytes=1 << 30)
        ids = [b.add(mesh, u0, dt=dt, nsteps=5, **m.physics()) for m, mesh, u0, dt in items]
        if tuned:
            b.tune_in_steps()
        b.advance(2)   # tuning continues across advance calls
        b.advance(3)
        if tuned:
            for m, mesh, _, _ in items:
                v, ms, lift_ms = b.class_info(mesh.dim, mesh.order, m.kind == "tgv")
                timed = [t for t in ms if t > 0]
                assert timed and ms[v] == min(timed)
                assert (lift_ms > 0) == (m.kind == "tgv")
        states.append([b.read(sid) for sid in ids])
        b.close()
    for a, c in zip(*states):
        assert np.array_equal(a, c)


def test_many_admissions_through_the_upload_ring_and_read_many():
    """Enough admissions that their geometry, neighbour tables and normals wrap
    the 32 MB pinned upload ring; the class tables go up once,
    before the first launches.  A sample of solves matches the FP64 plain path
    and read_many returns exactly what read returns."""
    ens = tgv_ensemble(160, n_range=(10, 12), orders=(2, 3), seed=7)   # ~53 MB of uploads
    items = _setup(ens, cfl=0.2)
    b = Batch("fp64", arena_bytes=4 << 30)
    ids = [b.add(mesh, u0, dt=dt, nsteps=2, **m.physics()) for m, mesh, u0, dt in items]
    b.advance(2)
    many = b.read_many(ids)
    for k in list(range(0, len(items), 23)) + [len(items) - 1]:
        m, mesh, u0, dt = items[k]
        assert np.array_equal(many[k], b.read(ids[k]))
        assert norm_err(many[k], plain(m, u0, dt, 2), mesh.num_fields) <= 1e-12
    b.close()


def test_add_many_matches_add_and_stops_at_a_bad_solve():
    """add_many prepares the solves on host threads and admits them in order:
    the states match one-by-one admission bit for bit; a solve whose mesh
    fails the checks stops the call there, the solves before it stay
    admitted and the ids from it on are -1."""
    from prandtl_b200._lib import PrandtlError
    items = _setup(MIX)
    spec = [(mesh, u0, dict(dt=dt, nsteps=3, **m.physics())) for m, mesh, u0, dt in items]
    b1 = Batch("fp32", arena_bytes=1 << 30)
    ids1 = [b1.add(mesh, u0, **kw) for mesh, u0, kw in spec]
    b2 = Batch("fp32", arena_bytes=1 << 30)
    ids2 = b2.add_many(spec)
    assert sorted(ids2) == sorted(set(ids2)) and min(ids2) >= 0
    b1.advance(3)
    b2.advance(3)
    for i1, i2 in zip(ids1, ids2):
        assert np.array_equal(b1.read(i1), b2.read(i2))
    b1.close()
    b2.close()
    # a mesh with a non-positive det J in the middle of the list
    bad_mesh, bad_u0, bad_kw = spec[1]
    import copy
    bad = copy.deepcopy(bad_mesh)
    bad.elem_detj[0] = -1.0
    b3 = Batch("fp32", arena_bytes=1 << 30)
    with pytest.raises(PrandtlError) as ei:
        b3.add_many([spec[0], (bad, bad_u0, bad_kw), spec[2]])
    assert "solve 1" in str(ei.value)
    b3.close()


def test_cfl_time_step_follows_lambda():
    m = Member("tgv", 3, 2, 0.2, 400.0)
    mesh = m.mesh()
    u0 = m.initial_state(mesh)
    b = Batch("fp64", arena_bytes=1 << 28)
    sid = b.add(mesh, u0, dt=1e-3, nsteps=3, cfl=0.4, **m.physics())
    b.advance(1)
    q = b.query(sid)
    # lambda of the step's stages is close to the state's max |V|+c
    from prandtl_b200.ensemble import max_char_speed
    assert abs(q["lambda_max"] / max_char_speed(u0, 3) - 1) < 1e-2
    assert q["dt"] == pytest.approx(0.4 * mesh.hmin / (q["lambda_max"] * 9), rel=1e-14)
    b.close()


def test_ensemble_members_small_sample():
    ens = tgv_ensemble(6, n_range=(2, 3))
    items = _setup(ens, cfl=0.2)
    b = Batch("fp64", arena_bytes=1 << 30)
    ids = [b.add(mesh, u0, dt=dt, nsteps=2, **m.physics()) for m, mesh, u0, dt in items]
    b.advance(2)
    for sid, (m, mesh, u0, dt) in zip(ids, items):
        assert norm_err(b.read(sid), plain(m, u0, dt, 2), mesh.num_fields) <= 1e-12
    b.close()


def test_blending_and_reference_mode_classes():
    """Classes with subcell-FV blending (2D Kelvin-Helmholtz) and the
    reference's own Navier-Stokes (quirks = reference: the gradient form) run in
    one batch next to fixed-mode solves and match the one-operator path."""
    from prandtl_b200.operator import DGSEMOperator
    kh = periodic_box(2, 8, 3, -1.0, 1.0)
    u_kh = cases.kelvin_helmholtz(kh)
    tg = periodic_box(3, 2, 3, 0.0, 2 * np.pi)
    u_tg = cases.taylor_green(tg)
    runs = [(kh, u_kh, dict(blending=True, quirks="fixed")),
            (kh, u_kh, dict(blending=True, quirks="reference")),
            (tg, u_tg, dict(parabolic=True, mu=1 / 1600, Pr=0.71, quirks="reference")),
            (tg, u_tg, dict(parabolic=True, mu=1 / 1600, Pr=0.71, quirks="fixed"))]
    b = Batch("fp64", "RK3SSP", arena_bytes=1 << 28)
    ids = []
    for mesh, u0, kw in runs:
        ids.append(b.add(mesh, u0, dt=fixed_dt(mesh, u0, 0.2), nsteps=3, **kw))
    b.advance(3)
    for sid, (mesh, u0, kw) in zip(ids, runs):
        op = DGSEMOperator(mesh, **kw)
        ref = u0.copy()
        op.Step(ref, fixed_dt(mesh, u0, 0.2), scheme="RK3SSP", nsteps=3)
        op.close()
        assert norm_err(b.read(sid), ref, mesh.num_fields) <= 1e-12, kw
    b.close()
