"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no unit tests or golden data for this path, so the oracle
is checked against the mathematical properties the discretisation must have
and, in test_ref_pin.py, against the reference's own sources compiled here.
"""
import numpy as np
import pytest

from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box, gauss_lobatto


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_gl_rule_and_derivative_matrix(oracle_mod, order):
    x, w, D = oracle_mod.gl(order)
    xm, wm = gauss_lobatto(order)
    np.testing.assert_allclose(x, xm, atol=1e-15)
    np.testing.assert_allclose(w, wm, atol=1e-15)
    assert abs(w.sum() - 1.0) < 1e-15
    for k in range(2 * order):     # GL is exact to degree 2N-1
        assert abs(np.dot(w, x ** k) - 1.0 / (k + 1)) < 1e-14
    for k in range(order + 1):     # D differentiates degree <= N exactly
        np.testing.assert_allclose(D @ x ** k, k * x ** max(k - 1, 0) if k else 0 * x, atol=1e-12)
    # summation-by-parts: W D + (W D)^T = diag(-1, 0, ..., 0, 1)
    Q = np.diag(w) @ D
    B = np.zeros_like(Q)
    B[0, 0], B[-1, -1] = -1.0, 1.0
    np.testing.assert_allclose(Q + Q.T, B, atol=1e-14)


def test_log_mean_branches(oracle_mod):
    L = oracle_mod.lib()
    rng = np.random.default_rng(0)
    for _ in range(200):
        x = rng.uniform(0.1, 10)
        for rel in (1e-9, 1e-6, 1e-3, 0.0199, 0.0201, 0.1, 1.0, 5.0):
            y = x * (1 + rel)
            X, Y = np.longdouble(x), np.longdouble(y)
            f = (Y - X) / (Y + X)
            if abs(f) < 0.3:   # (x+y)/2 / (atanh(f)/f), series in long double
                s, term, k = np.longdouble(0), np.longdouble(1), 0
                while abs(term) > 1e-25:
                    term = f ** (2 * k) / (2 * k + 1)
                    s += term
                    k += 1
                exact = (X + Y) / 2 / s
            else:
                exact = (Y - X) / np.log(Y / X)
            got = L.oracle_log_mean(x, y)
            assert abs(got - float(exact)) <= 2e-14 * float(exact)
            assert abs(L.oracle_log_mean(y, x) - got) <= 2e-14 * got
    assert L.oracle_log_mean(2.0, 2.0) == 2.0


def _flux_exact(dim, s, n, gamma=1.4):
    rho, m, E = s[0], np.asarray(s[1:1 + dim]), s[-1]
    v = m / rho
    p = (gamma - 1) * (E - 0.5 * rho * v @ v)
    vn = v @ n
    return np.concatenate([[rho * vn], m * vn + p * np.asarray(n), [(E + p) * vn]])


@pytest.mark.parametrize("dim", [2, 3])
def test_two_point_flux_consistency_and_symmetry(oracle_mod, dim):
    import ctypes as C
    L = oracle_mod.lib()
    dp = C.POINTER(C.c_double)
    rng = np.random.default_rng(dim)
    for _ in range(50):
        rho = rng.uniform(0.5, 2)
        v = rng.uniform(-1, 1, dim)
        p = rng.uniform(0.5, 2)
        s = np.concatenate([[rho], rho * v, [p / 0.4 + 0.5 * rho * v @ v]])
        n = rng.uniform(-1, 1, dim)
        F = np.empty(dim + 2)
        L.oracle_volume_flux(dim, 1.4, s.ctypes.data_as(dp), s.ctypes.data_as(dp),
                             n.ctypes.data_as(dp), n.ctypes.data_as(dp), F.ctypes.data_as(dp))
        np.testing.assert_allclose(F, _flux_exact(dim, s, n), rtol=1e-13, atol=1e-13)
        # face flux of equal states has zero dissipation
        G = np.empty(dim + 2)
        for q in (0, 1):
            L.oracle_face_flux(dim, 1.4, q, 1, s.ctypes.data_as(dp), s.ctypes.data_as(dp),
                               n.ctypes.data_as(dp), G.ctypes.data_as(dp))
            if dim == 2 or q == 1:
                np.testing.assert_allclose(G, F, rtol=1e-13, atol=1e-13)
        s2 = s * rng.uniform(0.9, 1.1, dim + 2)
        A, B = np.empty(dim + 2), np.empty(dim + 2)
        L.oracle_volume_flux(dim, 1.4, s.ctypes.data_as(dp), s2.ctypes.data_as(dp),
                             n.ctypes.data_as(dp), n.ctypes.data_as(dp), A.ctypes.data_as(dp))
        L.oracle_volume_flux(dim, 1.4, s2.ctypes.data_as(dp), s.ctypes.data_as(dp),
                             n.ctypes.data_as(dp), n.ctypes.data_as(dp), B.ctypes.data_as(dp))
        np.testing.assert_allclose(A, B, rtol=1e-12, atol=1e-15)


def test_q3_quirk_only_touches_3d_energy_dissipation(oracle_mod):
    import ctypes as C
    L = oracle_mod.lib()
    dp = C.POINTER(C.c_double)
    s1 = np.array([1.0, 0.1, 0.2, 0.3, 2.5])
    s2 = np.array([1.1, 0.2, 0.1, 0.4, 2.7])
    n = np.array([0.3, 0.4, 0.5])
    a, b = np.empty(5), np.empty(5)
    L.oracle_face_flux(3, 1.4, 0, 1, s1.ctypes.data_as(dp), s2.ctypes.data_as(dp), n.ctypes.data_as(dp), a.ctypes.data_as(dp))
    L.oracle_face_flux(3, 1.4, 1, 1, s1.ctypes.data_as(dp), s2.ctypes.data_as(dp), n.ctypes.data_as(dp), b.ctypes.data_as(dp))
    np.testing.assert_array_equal(a[:4], b[:4])
    assert a[4] != b[4]


def _entropy_vars(u, dim, gamma=1.4):
    nf = dim + 2
    U = u.reshape(nf, -1)
    rho = U[0]
    vel = U[1:1 + dim] / rho
    p = (gamma - 1) * (U[-1] - 0.5 * rho * np.sum(vel ** 2, 0))
    beta = rho / p
    s = np.log(p * rho ** -gamma)
    return np.concatenate([((gamma - s) / (gamma - 1) - beta * 0.5 * np.sum(vel ** 2, 0))[None],
                           beta * vel, -beta[None]])


def _mesh(dim, n=3, order=3, seed=1):
    rng = np.random.default_rng(seed)
    return periodic_box(dim, n, order, 0.0, 1.0, affine=np.eye(dim) + 0.15 * rng.uniform(-1, 1, (dim, dim)))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("phys", [dict(parabolic=0, blending=0), dict(parabolic=0, blending=1),
                                  dict(parabolic=1, blending=0, mu=0.01), dict(parabolic=1, blending=1, mu=0.01)])
def test_free_stream_preservation(oracle_mod, dim, phys):
    m = _mesh(dim)
    u = cases.free_stream(m, rho=1.3, vel=[0.3, -0.2, 0.4][:dim], p=0.9)
    d = oracle_mod.Oracle(m, quirks=1, **phys).rhs(u)["dudt"]
    assert np.abs(d).max() < 1e-12


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("par", [0, 1])
def test_conservation_and_entropy_conservation(oracle_mod, dim, par):
    m = _mesh(dim, n=4, seed=2)
    u = cases.perturbed(m, cases.free_stream(m), amp=0.2, seed=3)
    wJ = m.node_weights()
    d = oracle_mod.Oracle(m, quirks=1, surface_dissipation=0, parabolic=par, mu=0.0).rhs(u)["dudt"]
    D = d.reshape(m.num_fields, -1)
    for f in range(m.num_fields):
        assert abs(np.sum(wJ * D[f])) <= 1e-13 * np.sum(wJ * np.abs(D[f]))
    v = _entropy_vars(u, dim)
    assert abs(np.sum(wJ * np.sum(v * D, 0))) <= 1e-13 * np.sum(wJ * np.sum(np.abs(v * D), 0))


@pytest.mark.parametrize("dim", [2, 3])
def test_viscous_terms_dissipate_entropy(oracle_mod, dim):
    m = _mesh(dim, n=3, seed=5)
    u = cases.perturbed(m, cases.free_stream(m), amp=0.2, seed=6)
    wJ = m.node_weights()
    v = _entropy_vars(u, dim)
    d0 = oracle_mod.Oracle(m, quirks=1, surface_dissipation=0, parabolic=1, mu=0.0).rhs(u)["dudt"]
    d1 = oracle_mod.Oracle(m, quirks=1, surface_dissipation=0, parabolic=1, mu=0.01).rhs(u)["dudt"]
    S = lambda d: float(np.sum(wJ * np.sum(v * d.reshape(m.num_fields, -1), 0)))
    # d/dt of the entropy sum (-rho s/(gamma-1)) gets a non-positive viscous part
    assert S(d1) - S(d0) < 0


def test_reference_quirks_change_3d_ns_only(oracle_mod):
    m3 = _mesh(3, n=2)
    u3 = cases.perturbed(m3, cases.free_stream(m3, rho=1.3), amp=0.2, seed=1)
    a = oracle_mod.Oracle(m3, quirks=0, parabolic=1, mu=0.01).rhs(u3)["dudt"]
    b = oracle_mod.Oracle(m3, quirks=1, parabolic=1, mu=0.01).rhs(u3)["dudt"]
    assert np.abs(a - b).max() > 1e-3
    m2 = _mesh(2)
    u2 = cases.perturbed(m2, cases.free_stream(m2), amp=0.2, seed=1)
    a = oracle_mod.Oracle(m2, quirks=0).rhs(u2)["dudt"]
    b = oracle_mod.Oracle(m2, quirks=1).rhs(u2)["dudt"]
    np.testing.assert_array_equal(a, b)    # 2D Euler has no reference defect


def test_alpha_of_pure_top_mode(oracle_mod):
    """rho*p carrying only the highest Legendre mode gives eta = 1 -> alpha_max."""
    m = periodic_box(2, 2, 3, 0.0, 1.0)
    x, y = m.coords
    xi = (x % 0.5) / 0.5
    P3 = lambda t: 0.5 * (5 * (2 * t - 1) ** 3 - 3 * (2 * t - 1))
    rho = 1.0 + 0.0 * x
    p = 1.0 + 0.3 * P3(xi) * P3((y % 0.5) / 0.5)
    u = np.concatenate([rho, 0 * x, 0 * x, p / 0.4])
    a = oracle_mod.Oracle(m, blending=1, alpha_max=0.5).rhs(u, want_alpha=True)["alpha"]
    np.testing.assert_allclose(a, 0.5)
    u_smooth = np.concatenate([rho, 0 * x, 0 * x, (1.0 + 0.01 * x) / 0.4])
    a = oracle_mod.Oracle(m, blending=1).rhs(u_smooth, want_alpha=True)["alpha"]
    np.testing.assert_array_equal(a, 0.0)


@pytest.mark.parametrize("scheme", [0, 1])
def test_rk_order(oracle_mod, scheme):
    """Halving dt on the isentropic vortex reduces the step error at the scheme's order."""
    m = periodic_box(2, 4, 3, 0.0, 10.0)
    u0 = cases.isentropic_vortex(m)
    o = oracle_mod.Oracle(m)
    T = 0.05
    ref = o.step(u0, T / 64, scheme=1, nsteps=64)
    e1 = np.abs(o.step(u0, T / 4, scheme=scheme, nsteps=4) - ref).max()
    e2 = np.abs(o.step(u0, T / 8, scheme=scheme, nsteps=8) - ref).max()
    order = np.log2(e1 / e2)
    assert order > (2.6 if scheme == 0 else 3.6)


# ---------------------------------------------------------------- boundary faces
def _bdr_free_stream(oracle_mod, dim, kinds, vel):
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box
    sides = {2: [0, 1, 2, 3], 3: [0, 1, 2, 3, 4, 5]}[dim]
    mesh = periodic_box(dim, 3, 3, 0.0, 1.0, bcs=sides)
    u = cases.free_stream(mesh, rho=1.2, vel=vel, p=2.0)
    nf = dim + 2
    state = list(u.reshape(nf, -1)[:, 0])
    prim = [1.2] + list(vel) + [2.0]
    data = {"state": state, "riemann": prim, "inflow_rv": prim[:-1]}
    bcs = [(k, data.get(k), 2.0 if k == "pressure_outflow" else None) for k in kinds]
    return mesh, oracle_mod.Oracle(mesh, quirks=1, bcs=bcs).rhs(u)["dudt"]


@pytest.mark.parametrize("dim", [2, 3])
def test_boundary_free_stream_preserved(oracle_mod, dim):
    """A uniform state is kept by inflow of that state, outflow, pressure
    outflow at its pressure, Riemann invariants of that state and subsonic
    inflow of its density and velocity on every side."""
    for k in ("state", "outflow", "pressure_outflow", "riemann", "inflow_rv"):
        _, d = _bdr_free_stream(oracle_mod, dim, [k] * 2 * dim, [0.3, -0.2, 0.1][:dim])
        assert np.abs(d).max() < 1e-12, k


def test_wall_parallel_flow_preserved(oracle_mod):
    """Flow along x between slip walls (or symmetry planes) at y = 0, 1 is
    kept: zero normal velocity, the wall flux is the pressure flux."""
    for wall in ("slip_wall", "symmetry"):
        _, d = _bdr_free_stream(oracle_mod, 2, ["outflow", "outflow", wall, wall], [0.4, 0.0])
        assert np.abs(d).max() < 1e-12, wall


# ---------------------------------------------------------------- axisymmetric (z, r)
def test_axisymmetric_free_stream_and_recovery(oracle_mod):
    """Uniform axial flow between the axis and a slip wall is kept (the r-weighted
    pressure flux balances the source); off the axis U = rU / r exactly; on the
    axis the radial momentum and its rate are zero."""
    import ctypes as C
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box
    for N in (1, 2, 3, 4):
        mesh = periodic_box(2, (4, 3), N, (0.0, 0.0), (2.0, 1.0), bcs=[0, 0, 1, 2])
        bcs = [("outflow",), ("axis",), ("slip_wall",)]
        U = cases.free_stream(mesh, rho=1.2, vel=[0.3, 0.0], p=1.5).reshape(4, -1)
        r = mesh.coords[1]
        orc = oracle_mod.Oracle(mesh, quirks=1, bcs=bcs, axisymmetric=1)
        d = orc.rhs((U * r[None, :]).reshape(-1))["dudt"]
        assert np.abs(d).max() < 1e-12, N
        Up = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.2, vel=[0.3, 0.1], p=1.5), amp=0.1, seed=N)
        Up = Up.reshape(4, -1)
        rUp = (Up * r[None, :]).reshape(-1)
        rec = np.empty_like(rUp)
        dp = C.POINTER(C.c_double)
        assert oracle_mod.lib().oracle_recover_weighted(C.byref(orc.m), C.byref(orc.c), rUp.ctypes.data_as(dp),
                                                        rec.ctypes.data_as(dp)) == 0
        rec = rec.reshape(4, -1)
        off = r > 1e-14
        np.testing.assert_allclose(rec[:, off], Up[:, off], rtol=1e-14)
        assert (rec[2, ~off] == 0).all() and (rec[0, ~off] > 0).all()
        assert (orc.rhs(rUp)["dudt"].reshape(4, -1)[2, ~off] == 0).all()


def test_axisymmetric_density_floor_takes_the_nearest_node(oracle_mod):
    """Above the axis density floor (the reference's driver raises it to
    1e-8 rho_inf) the axis node copies the nearest off-axis node's U with zero
    radial momentum."""
    import ctypes as C
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box
    mesh = periodic_box(2, (3, 2), 3, (0.0, 0.0), (2.0, 1.0), bcs=[0, 0, 1, 2])
    bcs = [("outflow",), ("axis",), ("slip_wall",)]
    U = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.2, vel=[0.3, 0.1], p=1.5), amp=0.1, seed=3)
    r = mesh.coords[1]
    rU = (U.reshape(4, -1) * r[None, :]).reshape(-1)
    dp = C.POINTER(C.c_double)
    nd = (mesh.order + 1) ** 2
    for floor, copied in ((0.0, False), (100.0, True)):
        orc = oracle_mod.Oracle(mesh, quirks=1, bcs=bcs, axisymmetric=1, axis_rho_floor=floor)
        rec = np.empty_like(rU)
        assert oracle_mod.lib().oracle_recover_weighted(C.byref(orc.m), C.byref(orc.c), rU.ctypes.data_as(dp),
                                                        rec.ctypes.data_as(dp)) == 0
        rec = rec.reshape(4, -1)
        for g in np.flatnonzero(np.abs(r) <= 1e-14):
            e0 = (g // nd) * nd
            re = r[e0:e0 + nd]
            j = e0 + int(np.argmin(np.where(re > 0, re, np.inf)))
            want = U.reshape(4, -1)[:, j].copy()
            want[2] = 0.0
            assert np.allclose(rec[:, g], want, rtol=1e-14) == copied
