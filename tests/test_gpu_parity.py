"""CUDA path vs the CPU oracle, through the C ABI (marked gpu).

Tolerance: per-DOF normalised error (conftest.normalized_error) <= 1e-12 for
one RHS evaluation in FP64; trajectories <= 1e-10 after the stated steps.
"""
import numpy as np
import pytest

from conftest import normalized_error
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
TRAJ_TOL = 1e-10


def _op(mesh, **kw):
    from prandtl_b200.operator import DGSEMOperator
    return DGSEMOperator(mesh, **kw)


def _state(mesh, seed=0, amp=0.1):
    base = cases.free_stream(mesh, rho=1.2, vel=[0.4, -0.3, 0.2][: mesh.dim], p=1.5)
    return cases.perturbed(mesh, base, amp=amp, seed=seed)


def _affine(dim, seed=1):
    rng = np.random.default_rng(seed)
    return np.eye(dim) + 0.15 * rng.uniform(-1, 1, (dim, dim))


PHYS = [
    dict(parabolic=0, blending=0),
    dict(parabolic=0, blending=1),
    dict(parabolic=1, blending=0, mu=0.01, Pr=0.71),
    dict(parabolic=1, blending=1, mu=0.01, Pr=0.71),
]


@pytest.mark.parametrize("dim,n,order", [(2, 3, 3), (2, 2, 1), (2, 4, 2), (2, 2, 4), (2, 2, 5),
                                         (3, 2, 3), (3, 2, 1), (3, 3, 2), (3, 2, 4), (3, 2, 5), (3, 1, 3)])
@pytest.mark.parametrize("phys", range(len(PHYS)))
@pytest.mark.parametrize("quirks", ["reference", "fixed"])
def test_rhs_matches_oracle(oracle_mod, dim, n, order, phys, quirks):
    kw = PHYS[phys]
    mesh = periodic_box(dim, n, order, 0.0, 1.0, affine=_affine(dim))
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


def test_blending_active_kh(oracle_mod):
    """KH state on a coarse mesh: the indicator fires and FV blending is exercised."""
    mesh = periodic_box(2, 16, 3, -1.0, 1.0)
    u = cases.kelvin_helmholtz(mesh)
    ref = oracle_mod.Oracle(mesh, blending=1, alpha_max=0.5).rhs(u, want_alpha=True)
    assert (ref["alpha"] > 0).sum() > 0
    op = _op(mesh, blending=True, alpha_max=0.5)
    d = np.empty_like(u)
    op.Mult(u, d)
    assert normalized_error(d, ref["dudt"], 4) <= RHS_TOL
    np.testing.assert_allclose(op.alpha(), ref["alpha"], rtol=0, atol=1e-12)


def test_device_pointer_path_identical():
    torch = pytest.importorskip("torch")
    mesh = periodic_box(3, 3, 3, 0.0, 2 * np.pi)
    u = cases.taylor_green(mesh)
    op = _op(mesh, parabolic=True, mu=1 / 1600, Pr=0.71)
    d_host = np.empty_like(u)
    op.Mult(u, d_host)
    ut = torch.from_numpy(u).cuda()
    dt = torch.empty_like(ut)
    op.Mult(ut, dt)
    torch.cuda.synchronize()
    assert np.array_equal(dt.cpu().numpy(), d_host)


def test_deterministic():
    mesh = periodic_box(2, 8, 3, -1.0, 1.0)
    u = cases.kelvin_helmholtz(mesh)
    op = _op(mesh, blending=True)
    a, b = np.empty_like(u), np.empty_like(u)
    op.Mult(u, a)
    op.Mult(u, b)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("scheme", ["RK3SSP", "LSRK45"])
@pytest.mark.parametrize("case", ["ivortex", "tgv"])
def test_trajectory_matches_oracle(oracle_mod, scheme, case):
    if case == "ivortex":
        mesh = periodic_box(2, 8, 3, 0.0, 10.0)
        u0 = cases.isentropic_vortex(mesh)
        kw = dict(parabolic=0, blending=0)
        nsteps = 20
    else:
        mesh = periodic_box(3, 3, 3, 0.0, 2 * np.pi)
        u0 = cases.taylor_green(mesh)
        kw = dict(parabolic=1, blending=0, mu=1 / 1600, Pr=0.71)
        nsteps = 5
    orc = oracle_mod.Oracle(mesh, **kw)
    lam = orc.rhs(u0)["lambda_max"]
    dt = 0.5 * mesh.hmin / (lam * (mesh.order + 1) ** 2)
    ref = orc.step(u0, dt, scheme=0 if scheme == "RK3SSP" else 1, nsteps=nsteps)
    op = _op(mesh, **kw)
    u = u0.copy()
    op.Step(u, dt, scheme=scheme, nsteps=nsteps)
    assert normalized_error(u, ref, mesh.num_fields) <= TRAJ_TOL


def test_free_stream_preserved_gpu():
    """Fixed mode preserves a free stream on sheared meshes.  (Reference mode
    does not in 3D NS: its zeta-loop g/h mix-up breaks the metric identity;
    parity of that behaviour is covered by test_rhs_matches_oracle.)"""
    for dim in (2, 3):
        mesh = periodic_box(dim, 3, 3, 0.0, 1.0, affine=_affine(dim, 5))
        u = cases.free_stream(mesh)
        for kw in PHYS:
            op = _op(mesh, quirks="fixed", **kw)
            d = np.empty_like(u)
            op.Mult(u, d)
            assert np.abs(d).max() < 1e-12


def test_entropy_conservation_gpu():
    """Fixed mode, no surface dissipation, no blending: sum wJ v.dudt = 0."""
    for dim in (2, 3):
        mesh = periodic_box(dim, 4, 3, 0.0, 1.0, affine=_affine(dim, 7))
        u = _state(mesh, seed=4, amp=0.2)
        for par in (0, 1):
            op = _op(mesh, quirks="fixed", surface_dissipation=False, parabolic=bool(par), mu=0.0)
            d = np.empty_like(u)
            op.Mult(u, d)
            nf = mesh.num_fields
            U, D = u.reshape(nf, -1), d.reshape(nf, -1)
            rho = U[0]
            vel = U[1:1 + dim] / rho
            p = 0.4 * (U[-1] - 0.5 * rho * np.sum(vel ** 2, 0))
            beta = rho / p
            s = np.log(p * rho ** -1.4)
            v = np.concatenate([((1.4 - s) / 0.4 - beta * 0.5 * np.sum(vel ** 2, 0))[None],
                                beta * vel, -beta[None]])
            wJ = mesh.node_weights()
            ent = float(np.sum(wJ * np.sum(v * D, 0)))
            scale = float(np.sum(wJ * np.sum(np.abs(v * D), 0)))
            assert abs(ent) <= 1e-13 * scale
            for f in range(nf):
                assert abs(float(np.sum(wJ * D[f]))) <= 1e-13 * float(np.sum(wJ * np.abs(D[f])))


def test_bad_mesh_rejected():
    from prandtl_b200 import _lib
    mesh = periodic_box(2, 3, 3)
    mesh.face_elems = mesh.face_elems[:-1]
    with pytest.raises(_lib.PrandtlError) as ei:
        _op(mesh)
    assert ei.value.status == _lib.PRANDTL_EUNSUPPORTED


def test_rhs_matches_reference_golden():
    """GPU RHS vs the outputs of the reference's own sources (tests/golden)."""
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_golden
    gold = np.load(os.path.join(here, "golden", "reference_rhs.npz"))
    for name, dim, n, order, par, bl, amp, seed in make_golden.CASES:
        mesh, A, u = make_golden.case_inputs(dim, n, order, amp, seed)
        op = _op(mesh, parabolic=bool(par), blending=bool(bl), quirks="reference", **make_golden.PHYS)
        d = np.empty_like(u)
        op.Mult(u, d)
        err = normalized_error(d, gold[f"{name}/dudt"], mesh.num_fields)
        assert err <= RHS_TOL, f"{name}: {err:.3e}"
        np.testing.assert_allclose(op.alpha(), gold[f"{name}/alpha"], rtol=0, atol=1e-12)


def _checkerboard_state(mesh, seed):
    """Smooth flow in even elements, nodal noise in odd ones: the two 16-lane
    groups of a warp (elements 2k, 2k+1 of the 2D N = 2, 3 meshes) take the
    subcell FV branch in one element and skip it in the other.  (At N = 1 the
    indicator blends every element, so no warp diverges there.)"""
    nf, nd = mesh.num_fields, mesh.nodes_per_elem
    u = _state(mesh, seed=seed, amp=0.0).reshape(nf, -1).copy()
    rng = np.random.default_rng(seed)
    e = np.repeat(np.arange(mesh.num_elements), nd)
    rough = (e % 2) == 1
    u[0, rough] *= 1.0 + 0.4 * rng.uniform(-1, 1, rough.sum())
    u[-1, rough] *= 1.0 + 0.4 * rng.uniform(-1, 1, rough.sum())
    return u.reshape(-1)


@pytest.mark.parametrize("dim,n,order", [(2, 8, 3), (2, 8, 2)])
def test_blending_in_alternate_elements_of_a_warp(oracle_mod, dim, n, order):
    """Regression: lane groups narrower than a warp synchronise only their own
    lanes, so an element that runs the subcell FV phase while its warp-mate
    skips it (and exits) still orders its shared-memory accesses.  Repeated
    evaluations on states where every other element is blended must match the
    oracle every time."""
    mesh = periodic_box(dim, n, order, 0.0, 1.0)
    kw = dict(parabolic=0, blending=1)
    op = _op(mesh, quirks="reference", **kw)
    for seed in range(6):
        u = _checkerboard_state(mesh, seed)
        ref = oracle_mod.Oracle(mesh, quirks=0, **kw).rhs(u, want_alpha=True)
        alpha = ref["alpha"]
        assert (alpha[1::2] > 0).all() and (alpha[0::2] == 0).all()
        d = np.empty_like(u)
        for _ in range(5):
            op.Mult(u, d)
            assert normalized_error(d, ref["dudt"], mesh.num_fields) <= RHS_TOL
            np.testing.assert_allclose(op.alpha(), alpha, rtol=0, atol=1e-12)
    op.close()


@pytest.mark.parametrize("scheme", ["RK3SSP", "LSRK45"])
@pytest.mark.parametrize("device", [False, True])
def test_step_graph_replay_bit_identical(scheme, device):
    """prandtl_step replays a captured graph for runs of >= 8 steps: the same
    states as one launch sequence per step, and the same launch count."""
    mesh = periodic_box(2, 6, 3, 0.0, 1.0, affine=_affine(2))
    u0 = _state(mesh, seed=3, amp=0.2)
    op_a = _op(mesh, blending=True, quirks="fixed")
    op_b = _op(mesh, blending=True, quirks="fixed")
    dt = 1e-4
    if device:
        torch = pytest.importorskip("torch")
        ua, ub = torch.from_numpy(u0).cuda(), torch.from_numpy(u0).cuda()
    else:
        ua, ub = u0.copy(), u0.copy()
    op_a.Step(ua, dt, scheme=scheme, nsteps=13)   # 3 graph replays + 1 step launched directly
    for _ in range(13):
        op_b.Step(ub, dt, scheme=scheme, nsteps=1)
    op_a.synchronize()
    op_b.synchronize()
    a = ua.cpu().numpy() if device else ua
    b = ub.cpu().numpy() if device else ub
    assert np.array_equal(a, b)
    assert op_a.kernel_launches == op_b.kernel_launches
    op_a.Step(ua, dt, scheme=scheme, nsteps=8)    # the cached graph again
    op_b.Step(ub, dt, scheme=scheme, nsteps=8)
    op_a.synchronize()
    op_b.synchronize()
    a = ua.cpu().numpy() if device else ua
    b = ub.cpu().numpy() if device else ub
    assert np.array_equal(a, b)
