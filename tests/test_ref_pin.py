"""Pin of the CPU oracle against the reference's own DGSEM sources.

oracle/_ref holds the reference's DGSEMIntegrator.cpp, LiftingBR1.cpp,
ChandrashekarFlux.cpp, NavierStokesFlux.cpp, BasicOperations.cpp,
PerssonPeraireIndicator.cpp and ModalBasis.cpp compiled unmodified against an
MFEM stand-in (oracle/ref_harness).  tests/golden/reference_rhs.npz holds their
outputs on seeded cases (tests/golden/make_golden.py).  Tolerance: normalised
per-DOF error 1e-13 (different summation order only).
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

PIN_TOL = 1e-13
GOLDEN = np.load(os.path.join(HERE, "golden", "reference_rhs.npz"))


@pytest.mark.parametrize("case", make_golden.CASES, ids=[c[0] for c in make_golden.CASES])
def test_oracle_matches_reference_golden(oracle_mod, case):
    name, dim, n, order, par, bl, amp, seed = case
    mesh, A, u = make_golden.case_inputs(dim, n, order, amp, seed)
    np.testing.assert_array_equal(A, GOLDEN[f"{name}/affine"])
    np.testing.assert_array_equal(u, GOLDEN[f"{name}/u"])
    r = oracle_mod.Oracle(mesh, parabolic=par, blending=bl, quirks=0, **make_golden.PHYS).rhs(u, want_alpha=True)
    assert normalized_error(r["dudt"], GOLDEN[f"{name}/dudt"], mesh.num_fields) <= PIN_TOL
    np.testing.assert_allclose(r["alpha"], GOLDEN[f"{name}/alpha"], rtol=0, atol=1e-14)
    if bl:
        assert (r["alpha"] > 0).any(), "blending case must exercise the subcell FV path"


def _ref(oracle_mod):
    if not oracle_mod.ref_available():
        if not os.path.isdir(os.path.join(os.environ.get("REF", "/root/reference"), "src")):
            pytest.skip("reference sources not present on this host")
        oracle_mod.build_ref()
    return oracle_mod


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("par", [0, 1])
@pytest.mark.parametrize("bl", [0, 1])
@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_oracle_matches_reference_sources(oracle_mod, dim, par, bl, order):
    o = _ref(oracle_mod)
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box
    rng = np.random.default_rng(order + 7 * dim)
    A = np.eye(dim) + 0.15 * rng.uniform(-1, 1, (dim, dim))
    n = 2 if (dim == 3 and order > 3) else 3
    mesh = periodic_box(dim, n, order, 0.0, 1.0, affine=A)
    base = cases.free_stream(mesh, rho=1.1, vel=[0.2, 0.5, -0.3][:dim], p=1.3)
    u = cases.perturbed(mesh, base, amp=0.3 if bl else 0.1, seed=order)
    kw = dict(parabolic=par, blending=bl, mu=0.01, Pr=0.71)
    a = o.Oracle(mesh, quirks=0, **kw).rhs(u, want_alpha=True, want_grad=bool(par))
    b = o.RefOperator(mesh, **kw).rhs(u, want_alpha=True, want_grad=bool(par))
    assert normalized_error(a["dudt"], b["dudt"], mesh.num_fields) <= PIN_TOL
    np.testing.assert_allclose(a["alpha"], b["alpha"], rtol=0, atol=1e-14)
    if par:   # lifted primitive gradients (the reference's dudx/dudy/dudz)
        assert normalized_error(a["grad"], b["grad"], dim * mesh.num_fields) <= PIN_TOL


def test_periodic_self_neighbour_mesh(oracle_mod):
    """n = 1: every face joins an element to itself (MFEM Elem1/Elem2 rule)."""
    o = _ref(oracle_mod)
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box
    for dim in (2, 3):
        mesh = periodic_box(dim, 1, 3, 0.0, 1.0)
        u = cases.perturbed(mesh, cases.free_stream(mesh), amp=0.1, seed=2)
        for par in (0, 1):
            a = o.Oracle(mesh, quirks=0, parabolic=par, mu=0.01).rhs(u)["dudt"]
            b = o.RefOperator(mesh, parabolic=par, mu=0.01).rhs(u)["dudt"]
            assert normalized_error(a, b, mesh.num_fields) <= PIN_TOL


def test_golden_fixtures_come_from_the_reference(oracle_mod):
    o = _ref(oracle_mod)
    for name, dim, n, order, par, bl, amp, seed in make_golden.CASES:
        mesh, A, u = make_golden.case_inputs(dim, n, order, amp, seed)
        r = o.RefOperator(mesh, parabolic=par, blending=bl, **make_golden.PHYS).rhs(u)
        np.testing.assert_array_equal(r["dudt"], GOLDEN[f"{name}/dudt"])


# ---------------------------------------------------------------- boundary faces
GOLD_BDR = [(c, st) for st, (cs, _, _, _) in make_golden.BC_SETS.items() for c in cs]


@pytest.mark.parametrize("case,bset", GOLD_BDR, ids=[c[0] for c, _ in GOLD_BDR])
def test_oracle_boundary_matches_reference_golden(oracle_mod, case, bset):
    """Boundary integrators (state, outflow, slip wall, symmetry, pressure outflow
    with the reference's Q9 aliasing, Riemann invariants with Q10, subsonic
    inflows; in the Navier-Stokes form the no-slip walls, BR1 boundary lifting
    with Q12 and the viscous boundary fluxes) against the reference's outputs."""
    name, dim, n, order, bl, amp, seed = case
    _, bcs, sides, par = make_golden.BC_SETS[bset]
    mesh, _, u = make_golden.case_inputs(dim, n, order, amp, seed, bcs=sides[dim])
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_rhs.npz"))
    o = oracle_mod.Oracle(mesh, parabolic=par, blending=bl, quirks=0, bcs=bcs[dim], **make_golden.PHYS).rhs(u)
    assert normalized_error(o["dudt"], gold[f"{name}/dudt"], mesh.num_fields) <= 1e-13


BC_KINDS = ["state", "outflow", "slip_wall", "symmetry", "pressure_outflow", "riemann", "riemann_supersonic",
            "inflow_rv", "inflow_pttt"]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", [1, 2, 4])
@pytest.mark.parametrize("kind", BC_KINDS)
def test_oracle_boundary_matches_reference_sources(oracle_mod, dim, order, kind):
    """One boundary condition on every bounded side, oracle vs the reference's
    boundary integrator compiled from its own sources."""
    if kind == "inflow_pttt" and dim == 3:
        pytest.skip("the reference's 3D SubsonicInflowPtTtAng writes past its direction vector")
    _ref(oracle_mod)
    bcs = [make_golden.bc_example(kind, dim)]
    sides = [0, 0, 0, 0] if dim == 2 else [0, 0, None, None, 0, 0]
    mesh = periodic_box(dim, 2, order, 0.0, 1.0, bcs=sides, affine=np.eye(dim) + 0.1 * np.eye(dim, k=1))
    base = cases.free_stream(mesh, rho=1.1, vel=[0.35, -0.2, 0.1][:dim], p=1.6)
    u = cases.perturbed(mesh, base, amp=0.2, seed=order)
    o = oracle_mod.Oracle(mesh, quirks=0, bcs=bcs).rhs(u)["dudt"]
    r = oracle_mod.RefOperator(mesh, quirks=0, bcs=bcs).rhs(u)["dudt"]
    assert normalized_error(o, r, mesh.num_fields) <= 1e-13


NS_KINDS = ["noslip_adiabatic", "noslip_isothermal", "outflow", "state", "pressure_outflow", "inflow_rv"]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", [1, 2, 4])
@pytest.mark.parametrize("bl", [0, 1])
@pytest.mark.parametrize("kind", NS_KINDS)
def test_oracle_ns_boundary_matches_reference_sources(oracle_mod, dim, order, bl, kind):
    """Navier-Stokes: one condition on every bounded side; lifting and viscous
    boundary terms of the reference's integrators compiled from its sources."""
    _ref(oracle_mod)
    bcs = [make_golden.bc_example(kind, dim)]
    sides = [0, 0, 0, 0] if dim == 2 else [0, 0, None, None, 0, 0]
    mesh = periodic_box(dim, 2, order, 0.0, 1.0, bcs=sides, affine=np.eye(dim) + 0.1 * np.eye(dim, k=1))
    base = cases.free_stream(mesh, rho=1.1, vel=[0.35, -0.2, 0.1][:dim], p=1.6)
    u = cases.perturbed(mesh, base, amp=0.2, seed=order)
    kw = dict(parabolic=1, blending=bl, quirks=0, bcs=bcs, **make_golden.PHYS)
    o = oracle_mod.Oracle(mesh, **kw).rhs(u, want_grad=True)
    r = oracle_mod.RefOperator(mesh, **kw).rhs(u, want_grad=True)
    assert normalized_error(o["dudt"], r["dudt"], mesh.num_fields) <= 1e-13
    assert normalized_error(o["grad"], r["grad"], mesh.num_fields * dim) <= 1e-13


def test_oracle_rejects_ns_boundaries_without_viscous_treatment(oracle_mod):
    mesh = periodic_box(2, 2, 2, 0.0, 1.0, bcs=[0, 0, None, None])
    u = cases.free_stream(mesh)
    for kind in ("slip_wall", "symmetry", "inflow_pttt"):
        with pytest.raises(RuntimeError):
            oracle_mod.Oracle(mesh, parabolic=1, bcs=[make_golden.bc_example(kind, 2)]).rhs(u)
    with pytest.raises(RuntimeError):   # Q13: reference-mode Riemann lifting is undefined
        oracle_mod.Oracle(mesh, parabolic=1, quirks=0, bcs=[make_golden.bc_example("riemann", 2)]).rhs(u)
    oracle_mod.Oracle(mesh, parabolic=1, quirks=1, bcs=[make_golden.bc_example("riemann", 2)]).rhs(u)


def test_reference_riemann_lifting_reads_an_unset_normal(oracle_mod):
    """Q13 as observed: the reference's NS operator with a Riemann-invariant
    boundary returns non-finite values (its lifting normalises a zero normal)."""
    _ref(oracle_mod)
    mesh = periodic_box(2, 2, 2, 0.0, 1.0, bcs=[0, 0, 0, 0])
    u = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.1, vel=[0.35, -0.2], p=1.6), amp=0.2, seed=1)
    r = oracle_mod.RefOperator(mesh, parabolic=1, bcs=[make_golden.bc_example("riemann", 2)]).rhs(u)
    assert not np.isfinite(r["dudt"]).all()


# ---------------------------------------------------------------- axisymmetric (z, r)
def _axi_case(order, blending, seed, n=(4, 3)):
    mesh = periodic_box(2, n, order, (0.0, 0.0), (2.0, 1.0), bcs=[0, 1, 2, 3],
                        affine=np.array([[1.0, 0.1], [0.0, 1.0]]))
    bcs = [("state", [1.3, 0.5, 0.0, 2.9]), ("outflow",), ("axis",), ("slip_wall",)]
    U = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.2, vel=[0.3, 0.05], p=1.5),
                        amp=0.3 if blending else 0.1, seed=seed).reshape(4, -1)
    return mesh, bcs, (U * mesh.coords[1][None, :]).reshape(-1)


@pytest.mark.parametrize("order", [1, 2, 3, 4])
@pytest.mark.parametrize("bl", [0, 1])
def test_oracle_axisymmetric_matches_reference_sources(oracle_mod, order, bl):
    """r-weighted volume, face, boundary and subcell-FV fluxes and the pressure
    source against the reference's integrators built with AXISYMMETRIC (both
    evaluated on the U the oracle recovers from r U)."""
    _ref(oracle_mod)
    mesh, bcs, rU = _axi_case(order, bl, order)
    kw = dict(quirks=0, bcs=bcs, axisymmetric=1, blending=bl)
    o = oracle_mod.Oracle(mesh, **kw).rhs(rU)["dudt"]
    r = oracle_mod.RefOperator(mesh, **kw).rhs(rU)["dudt"]
    assert normalized_error(o, r, 4) <= 1e-13


@pytest.mark.parametrize("case", make_golden.AXI_CASES, ids=[c[0] for c in make_golden.AXI_CASES])
def test_oracle_axisymmetric_matches_reference_golden(oracle_mod, case):
    """The committed outputs of the reference's AXISYMMETRIC build (runs on any
    host: no reference sources needed)."""
    name, n, order, bl, amp, seed = case
    mesh, u = make_golden.axi_inputs(n, order, bl, amp, seed)
    np.testing.assert_array_equal(u, GOLDEN[f"{name}/u"])
    r = oracle_mod.Oracle(mesh, quirks=0, blending=bl, bcs=make_golden.AXI_BCS, axisymmetric=1).rhs(u, want_alpha=True)
    assert normalized_error(r["dudt"], GOLDEN[f"{name}/dudt"], mesh.num_fields) <= PIN_TOL
    np.testing.assert_allclose(r["alpha"], GOLDEN[f"{name}/alpha"], rtol=0, atol=1e-14)
    if bl:
        assert (r["alpha"] > 0).any()


# ---------------------------------------------------------------- multilinear (non-affine) elements
@pytest.mark.parametrize("case", make_golden.CURVED_CASES, ids=[c[0] for c in make_golden.CURVED_CASES])
def test_oracle_curved_matches_reference_golden(oracle_mod, case):
    """Per-node metrics in the volume flux averages, per-node J, subcell metrics
    integrated along each line, per-face-node normals and J on both sides
    (DGSEMIntegrator.cpp:254-267, :1199-1304; LiftingBR1.cpp:40-49, :184-186):
    the oracle against the committed outputs of the reference's sources."""
    name, dim, n, order, par, bl, amp, seed, bset = case
    mesh, u = make_golden.curved_inputs(dim, n, order, amp, seed, bset)
    assert not mesh.affine
    np.testing.assert_array_equal(u, GOLDEN[f"{name}/u"])
    bcs = make_golden.BC_SETS[bset][1][dim] if bset else None
    r = oracle_mod.Oracle(mesh, parabolic=par, blending=bl, quirks=0, bcs=bcs, **make_golden.PHYS).rhs(u, want_alpha=True)
    assert normalized_error(r["dudt"], GOLDEN[f"{name}/dudt"], mesh.num_fields) <= PIN_TOL
    np.testing.assert_allclose(r["alpha"], GOLDEN[f"{name}/alpha"], rtol=0, atol=1e-14)
    if bl:
        assert (r["alpha"] > 0).any()


@pytest.mark.parametrize("case", make_golden.CURVED_AXI_CASES, ids=[c[0] for c in make_golden.CURVED_AXI_CASES])
def test_oracle_curved_axisymmetric_matches_reference_golden(oracle_mod, case):
    name, n, order, bl, amp, seed = case
    mesh, u = make_golden.curved_axi_inputs(n, order, bl, amp, seed)
    np.testing.assert_array_equal(u, GOLDEN[f"{name}/u"])
    r = oracle_mod.Oracle(mesh, quirks=0, blending=bl, bcs=make_golden.AXI_BCS, axisymmetric=1).rhs(u, want_alpha=True)
    assert normalized_error(r["dudt"], GOLDEN[f"{name}/dudt"], mesh.num_fields) <= PIN_TOL


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("par", [0, 1])
@pytest.mark.parametrize("bl", [0, 1])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_oracle_curved_matches_reference_sources(oracle_mod, dim, par, bl, order):
    o = _ref(oracle_mod)
    mesh = periodic_box(dim, 3, order, 0.0, 1.0, warp=make_golden.warp_field(dim, 0.05 + 0.01 * order))
    base = cases.free_stream(mesh, rho=1.1, vel=[0.2, 0.5, -0.3][:dim], p=1.3)
    u = cases.perturbed(mesh, base, amp=0.3 if bl else 0.1, seed=order)
    kw = dict(parabolic=par, blending=bl, mu=0.01, Pr=0.71)
    a = o.Oracle(mesh, quirks=0, **kw).rhs(u, want_alpha=True, want_grad=bool(par))
    b = o.RefOperator(mesh, **kw).rhs(u, want_alpha=True, want_grad=bool(par))
    assert normalized_error(a["dudt"], b["dudt"], mesh.num_fields) <= PIN_TOL
    np.testing.assert_allclose(a["alpha"], b["alpha"], rtol=0, atol=1e-14)
    if par:
        assert normalized_error(a["grad"], b["grad"], dim * mesh.num_fields) <= PIN_TOL


@pytest.mark.parametrize("order", [1, 2, 4])
@pytest.mark.parametrize("kind", ["state", "outflow", "slip_wall", "symmetry", "riemann", "inflow_rv"])
def test_oracle_curved_boundary_matches_reference_sources(oracle_mod, order, kind):
    """Boundary faces of multilinear elements: the face-node normals and J."""
    _ref(oracle_mod)
    bcs = [make_golden.bc_example(kind, 2)]
    mesh = periodic_box(2, 3, order, 0.0, 1.0, bcs=[0, 0, 0, 0], warp=make_golden.warp_field(2, 0.06))
    u = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.1, vel=[0.35, -0.2], p=1.6), amp=0.2, seed=order)
    o = oracle_mod.Oracle(mesh, quirks=0, bcs=bcs).rhs(u)["dudt"]
    r = oracle_mod.RefOperator(mesh, quirks=0, bcs=bcs).rhs(u)["dudt"]
    assert normalized_error(o, r, mesh.num_fields) <= 1e-13


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("bl", [0, 1])
def test_oracle_curved_axisymmetric_matches_reference_sources(oracle_mod, order, bl):
    _ref(oracle_mod)
    mesh, u = make_golden.curved_axi_inputs((4, 3), order, bl, 0.3 if bl else 0.1, order)
    kw = dict(quirks=0, bcs=make_golden.AXI_BCS, axisymmetric=1, blending=bl)
    o = oracle_mod.Oracle(mesh, **kw).rhs(u)["dudt"]
    r = oracle_mod.RefOperator(mesh, **kw).rhs(u)["dudt"]
    assert normalized_error(o, r, 4) <= 1e-13


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 3), (3, 2), (3, 3)])
def test_oracle_curved_free_stream(oracle_mod, dim, order):
    """A uniform state on multilinear elements stays uniform (the metric
    identities hold for the nodal adjugates: 2D for N >= 1, 3D for N >= 2)."""
    mesh = periodic_box(dim, 3, order, 0.0, 1.0, warp=make_golden.warp_field(dim, 0.06))
    u = cases.free_stream(mesh, rho=1.2, vel=[0.3, -0.2, 0.1][:dim], p=1.5)
    for par in (0, 1):
        d = oracle_mod.Oracle(mesh, quirks=1, parabolic=par).rhs(u)["dudt"]
        assert np.abs(d).max() < 1e-12


@pytest.mark.parametrize("order,nx,ny", [(1, 12, 6), (2, 8, 4)])
def test_oracle_ramp_matches_reference_sources(oracle_mod, order, nx, ny):
    """The reference's axisymmetric Ramp case geometry (trapezoidal cells over
    the cone, inflow / outflow / axis / slip-wall boundaries, blending) through
    the reference's own integrators."""
    _ref(oracle_mod)
    mesh = cases.ramp_mesh(order, nx, ny)
    U = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.0, vel=[2.0, 0.0], p=1 / 1.4),
                        amp=0.3, seed=order).reshape(4, -1)
    rU = (U * mesh.coords[1][None, :]).reshape(-1)
    kw = dict(quirks=0, bcs=cases.RAMP_BCS, axisymmetric=1, blending=1)
    o = oracle_mod.Oracle(mesh, **kw).rhs(rU, want_alpha=True)
    r = oracle_mod.RefOperator(mesh, **kw).rhs(rU, want_alpha=True)
    assert normalized_error(o["dudt"], r["dudt"], 4) <= 1e-13
    np.testing.assert_allclose(o["alpha"], r["alpha"], rtol=0, atol=1e-14)
