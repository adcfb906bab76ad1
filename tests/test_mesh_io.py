"""Mesh ingestion (prandtl_mesh_read): MFEM v1.0 and Gmsh 2.2 ASCII meshes.

The reader re-orients elements so that neighbouring faces are aligned, so a
read mesh and the generated box with the same cells differ by per-element
frames (node orders).  The checks therefore compare operator outputs node by
node, matched by (element centroid, node coordinate): the oracle's RHS on the
read mesh equals its RHS on the generated mesh.
"""
import os

import numpy as np
import pytest

from conftest import normalized_error
from prandtl_b200 import _lib
from prandtl_b200.mesh import periodic_box, read_mesh

HERE = os.path.dirname(os.path.abspath(__file__))
MESHES = os.path.join(HERE, "golden", "meshes")
SHEAR2 = np.array([[1.0, 0.2], [0.0, 1.1]])
SHEAR3 = np.array([[1.0, 0.1, 0.0], [0.0, 1.05, 0.15], [0.05, 0.0, 0.95]])
# the reference checkout (REF, as for oracle/ref_harness/build_ref.sh)
REF_CASES = os.path.join(os.environ.get("REF", "/root/reference"), "TestCases")


def smooth_state(mesh):
    x = mesh.coords
    dim = mesh.dim
    rho = 1.2 + 0.1 * np.sin(2.0 * x[0]) * np.cos(3.0 * x[1])
    vel = [0.3 + 0.05 * np.cos(2.0 * x[1]), -0.2 + 0.05 * np.sin(x[0]), 0.1 + 0.0 * x[0]][:dim]
    if dim == 3:
        rho = rho + 0.05 * np.sin(2.0 * x[2])
    p = 1.5 + 0.1 * np.cos(x[0] + x[1])
    E = p / 0.4 + 0.5 * rho * sum(v * v for v in vel)
    return np.concatenate([rho, *[rho * v for v in vel], E])


def node_index(mesh):
    """(rounded element centroid, rounded node coordinate) -> dof index."""
    E, ND, dim = mesh.num_elements, mesh.nodes_per_elem, mesh.dim
    X = mesh.coords.reshape(dim, E, ND)
    cen = X.mean(axis=2)
    out = {}
    for e in range(E):
        c = tuple(np.round(cen[:, e], 9))
        for n in range(ND):
            out[(c, tuple(np.round(X[:, e, n], 9)))] = e * ND + n
    return out


def matched(read, box, vals_read, vals_box):
    """Values of the read mesh, reordered to the box mesh's dofs."""
    ir, ib = node_index(read), node_index(box)
    assert ir.keys() == ib.keys()
    nf = read.num_fields
    perm = np.empty(read.ndof, dtype=np.int64)
    for k, j in ib.items():
        perm[j] = ir[k]
    return vals_read.reshape(nf, -1)[:, perm].reshape(-1), vals_box


def test_mfem_periodic_mesh_equals_generated_box(oracle_mod):
    """MFEM periodic form (identified vertices + L2 corner nodes): same
    elements, faces, normals and node coordinates as the generated box."""
    m = read_mesh(os.path.join(MESHES, "periodic_4x3.mesh"), 3)
    b = periodic_box(2, (4, 3), 3, (0.0, 0.0), (2.0, 1.5), affine=SHEAR2)
    np.testing.assert_allclose(m.elem_adj, b.elem_adj, rtol=0, atol=1e-14)
    np.testing.assert_allclose(m.elem_detj, b.elem_detj, rtol=1e-14)
    np.testing.assert_allclose(m.coords, b.coords, rtol=0, atol=1e-13)
    fm = {tuple(f): tuple(n) for f, n in zip(m.face_elems.tolist(), np.round(m.face_nor, 12).tolist())}
    fb = {tuple(f): tuple(n) for f, n in zip(b.face_elems.tolist(), np.round(b.face_nor, 12).tolist())}
    assert fm == fb
    assert m.hmin == pytest.approx(b.hmin, rel=1e-12)
    u = smooth_state(m)
    rm = oracle_mod.Oracle(m, quirks=1, parabolic=1, mu=0.01).rhs(u)["dudt"]
    rb = oracle_mod.Oracle(b, quirks=1, parabolic=1, mu=0.01).rhs(u)["dudt"]
    assert normalized_error(rm, rb, 4) <= 1e-14


CAVITY_EULER = [("state", [1.3, 0.5, 0.2, 2.9]), ("outflow",), ("slip_wall",), ("pressure_outflow", None, 1.4)]
CAVITY_NS = [("noslip_adiabatic", dict(wall_vel=[0.0, 0.0], heat_flux=0.0)), ("outflow",),
             ("noslip_isothermal", dict(wall_vel=[0.0, 0.0], wall_T=0.0045)),
             ("noslip_adiabatic", dict(wall_vel=[1.0, 0.0], heat_flux=0.01))]


@pytest.mark.parametrize("refine", [0, 1])
@pytest.mark.parametrize("hilbert", [False, True])
@pytest.mark.parametrize("physics", ["euler", "ns"])
def test_gmsh_cavity_matches_generated_box(oracle_mod, refine, hilbert, physics):
    """Gmsh quads listed from random corners (re-oriented on reading), named
    boundary groups, uniform refinement and Hilbert order: the oracle RHS on
    the read mesh equals the RHS on the generated bounded box."""
    m = read_mesh(os.path.join(MESHES, "cavity_6x5.msh"), 3, refine=refine, hilbert=hilbert)
    n = (6 << refine, 5 << refine)
    b = periodic_box(2, n, 3, (0.0, 0.0), (1.0, 1.0), affine=SHEAR2, bcs=[0, 1, 2, 3])
    assert m.num_elements == b.num_elements and m.num_faces == b.num_faces
    assert (m.elem_detj > 0).all()
    bcs = CAVITY_EULER if physics == "euler" else CAVITY_NS
    kw = dict(quirks=1, bcs=bcs) if physics == "euler" else dict(quirks=1, bcs=bcs, parabolic=1, mu=0.01, R_gas=287.05)
    rm = oracle_mod.Oracle(m, **kw).rhs(smooth_state(m))["dudt"]
    rb = oracle_mod.Oracle(b, **kw).rhs(smooth_state(b))["dudt"]
    a, r = matched(m, b, rm, rb)
    assert normalized_error(a, r, 4) <= 1e-12


@pytest.mark.parametrize("quirks,blending", [(0, 0), (1, 0), (1, 1)])
def test_gmsh_hex_channel_matches_generated_box(oracle_mod, quirks, blending):
    """Hexahedra listed from random proper rotations of their corners.  (The
    reference's 3D face flux with quirks = 0 is not antisymmetric (Q3), so its
    subcell-FV lines, which run along each element's local axes, depend on the
    element frame: reference mode with blending is compared on unrotated
    frames only.)"""
    m = read_mesh(os.path.join(MESHES, "channel_4x3x2.msh"), 2)
    b = periodic_box(3, (4, 3, 2), 2, (0.0, 0.0, 0.0), (2.0, 1.0, 1.0), affine=SHEAR3, bcs=[0, 1, 2, 3, 4, 5])
    bcs = [("state", [1.3, 0.5, 0.2, -0.1, 2.9]), ("outflow",), ("slip_wall",), ("symmetry",),
           ("pressure_outflow", None, 1.4), ("outflow",)]
    kw = dict(bcs=bcs, blending=blending, quirks=quirks)
    rm = oracle_mod.Oracle(m, **kw).rhs(smooth_state(m))["dudt"]
    rb = oracle_mod.Oracle(b, **kw).rhs(smooth_state(b))["dudt"]
    a, r = matched(m, b, rm, rb)
    assert normalized_error(a, r, 5) <= 1e-11


def test_boundary_names_map_to_conditions():
    path = os.path.join(MESHES, "cavity_6x5.msh")
    m = read_mesh(path, 2)
    bf = m.face_elems[:, 2] < 0
    assert sorted(set(m.face_attr[bf].tolist())) == [1, 2, 3, 4]
    assert (m.face_elems[bf, 3] == m.face_attr[bf] - 1).all()   # default: attribute - 1
    m2 = read_mesh(path, 2, boundary_conditions={"lid": 0, "left": 1, "right": 1, 3: 2})
    want = {4: 0, 1: 1, 2: 1, 3: 2}
    assert all(m2.face_elems[f, 3] == want[m2.face_attr[f]] for f in np.nonzero(bf)[0])
    assert (m2.face_attr[~bf] == 0).all() and (m2.elem_attr == 5).all()
    with pytest.raises(KeyError):
        read_mesh(path, 2, boundary_conditions={"nozzle": 0})


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


GMSH_HEAD = "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n"


def test_rejected_meshes(tmp_path):
    def code(path):
        with pytest.raises(_lib.PrandtlError) as ei:
            read_mesh(path, 2)
        return ei.value.status, str(ei.value)

    tri = _write(tmp_path, "tri.msh", GMSH_HEAD + "$Nodes\n3\n1 0 0 0\n2 1 0 0\n3 0 1 0\n$EndNodes\n"
                 "$Elements\n1\n1 2 2 1 1 1 2 3\n$EndElements\n")
    assert code(tri)[0] == _lib.PRANDTL_EUNSUPPORTED
    # three quads around a vertex: no aligned frames exist
    star = _write(tmp_path, "star.msh", GMSH_HEAD + "$Nodes\n7\n1 0 0 0\n2 1 0 0\n3 0.5 0.866 0\n"
                  "4 -0.5 0.866 0\n5 -0.5 -0.866 0\n6 0.5 -0.866 0\n7 -1 0 0\n$EndNodes\n"
                  "$Elements\n3\n1 3 2 1 1 1 2 3 4\n2 3 2 1 1 1 4 7 5\n3 3 2 1 1 1 5 6 2\n$EndElements\n")
    st, msg = code(star)
    assert st == _lib.PRANDTL_EUNSUPPORTED
    v4 = _write(tmp_path, "v4.msh", "$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
    assert code(v4)[0] == _lib.PRANDTL_EUNSUPPORTED
    assert code(str(tmp_path / "missing.msh"))[0] == _lib.PRANDTL_EINVAL


REF_MESHES = {   # file -> (elements, boundary faces) as read at refine 0, or the rejection text
    "Euler/2D/IsentropicVortex/IsentropicVortex.mesh": (9, 0),
    "Euler/2D/KelvinHelmholtzInstability/KelvinHelmholtzInstability.mesh": (9, 0),
    "NavierStokes/2D/LidDrivenCavity/LidDrivenCavity.msh": (256, 64),
    "Euler/2D/ForwardFacingStep/ForwardFacingStep.msh": (3400, 260),
    "Euler/2D/DoubleMachReflection/DoubleMachReflection.msh": (36864, 960),
    "Euler/2D/BackwardFacingStep/BackwardFacingStep.msh": (35000, 800),
    "Euler/2D/Ramp/Ramp15deg_v2.msh": (4802, 294),
    "Euler/2D/Nagashima_Ramjet/TR0/Nagashima_TR0_10kQuad_v2.msh": "structured topology",
}


@pytest.mark.parametrize("rel", sorted(REF_MESHES))
def test_reference_test_case_meshes(rel):
    path = os.path.join(REF_CASES, rel)
    if not os.path.exists(path):
        pytest.skip("reference test cases not present on this host")
    want = REF_MESHES[rel]
    if isinstance(want, str):
        with pytest.raises(_lib.PrandtlError) as ei:
            read_mesh(path, 3)
        assert want in str(ei.value)
        return
    m = read_mesh(path, 3)
    assert (m.num_elements, int((m.face_elems[:, 2] < 0).sum())) == want
    assert (m.elem_detj > 0).all()
    if rel.endswith("Ramp15deg_v2.msh"):   # quadrilaterals over the ramp are not parallelograms
        assert not m.affine and (m.node_detj > 0).all()
    if rel.endswith("IsentropicVortex.mesh"):   # the 3x3 periodic [-1, 1]^2 box
        b = periodic_box(2, 3, 3, -1.0, 1.0)
        np.testing.assert_allclose(m.coords, b.coords, rtol=0, atol=1e-8)
    if rel.endswith("LidDrivenCavity.msh"):
        m2 = read_mesh(path, 3, boundary_conditions={"lid": 0, "left": 1, "right": 1, "bottom": 1})
        lid = m2.face_elems[(m2.face_elems[:, 2] < 0) & (m2.face_elems[:, 3] == 0)]
        assert len(lid) == 16


def test_gmsh_trapezoid_is_multilinear(tmp_path):
    """A quadrilateral that is not a parallelogram: the reader returns the
    multilinear map's geometry at every node (the same as the Python
    multilinear_geometry of its corners), per-face-node normals and the centre
    Jacobian's values per element."""
    from prandtl_b200.mesh import multilinear_geometry
    trap = _write(tmp_path, "trap.msh", GMSH_HEAD + "$Nodes\n4\n1 0 0 0\n2 2 0 0\n3 1.5 1 0\n4 0 1 0\n$EndNodes\n"
                  "$Elements\n1\n1 3 2 1 1 1 2 3 4\n$EndElements\n")
    m = read_mesh(trap, 3)
    assert not m.affine
    corners = np.array([[[0.0, 0.0], [2.0, 0.0], [0.0, 1.0], [1.5, 1.0]]])
    xy, adj, detj = multilinear_geometry(corners, m.nodes_1d)
    np.testing.assert_allclose(m.coords, xy, rtol=0, atol=1e-15)
    np.testing.assert_allclose(m.node_adj, adj, rtol=0, atol=1e-15)
    np.testing.assert_allclose(m.node_detj, detj, rtol=0, atol=1e-15)
    assert m.face_node_nor.shape == (4, 4, 2)
    # boundary face normals: outward, |n| = edge length; left edge x = 0 points to -x
    left = [f for f in range(4) if m.face_elems[f, 1] == 0][0]
    np.testing.assert_allclose(m.face_node_nor[left], np.tile([-1.0, 0.0], (4, 1)), atol=1e-15)
    assert m.hmin > 0


def test_multilinear_refinement_keeps_the_geometry(tmp_path):
    """Refining a multilinear element splits it in reference coordinates: the
    children's node coordinates lie on the parent's map."""
    trap = _write(tmp_path, "trap.msh", GMSH_HEAD + "$Nodes\n4\n1 0 0 0\n2 2 0 0\n3 1.5 1 0\n4 0 1 0\n$EndNodes\n"
                  "$Elements\n1\n1 3 2 1 1 1 2 3 4\n$EndElements\n")
    m = read_mesh(trap, 2, refine=1)
    assert m.num_elements == 4 and not m.affine
    area = (m.node_weights()).sum()
    assert area == pytest.approx(1.75, rel=1e-14)   # (2 + 1.5) / 2 * 1


@pytest.mark.parametrize("name,order,measure", [("bump_8x4.msh", 3, None), ("warped_3x3x2.msh", 2, 2.0)])
@pytest.mark.parametrize("refine,hilbert", [(0, False), (1, True), (2, False)])
def test_multilinear_fixture_meshes(name, order, measure, refine, hilbert):
    """Gmsh meshes of non-affine elements listed from random corner rotations:
    read with multilinear geometry, positive det J at every node, the domain
    measure kept by refinement, and face-node normals that are the elements'
    adjugate rows on both sides of every interior face."""
    m = read_mesh(os.path.join(MESHES, name), order, refine=refine, hilbert=hilbert)
    assert not m.affine and (m.node_detj > 0).all()
    area = m.node_weights().sum()
    if measure is None:   # the bump channel: 2 minus the area under the piecewise-linear floor
        xs = np.linspace(0.0, 2.0, 9)
        floor = 0.12 * np.sin(np.pi * np.clip(xs - 0.5, 0.0, 1.0)) ** 2
        measure = 2.0 - np.trapezoid(floor, xs)
    assert area == pytest.approx(measure, rel=1e-13)
    from prandtl_b200.mesh import face_node
    dim, Np = m.dim, m.order + 1
    for fc in range(m.num_faces):
        e1, l1, e2, l2 = (int(v) for v in m.face_elems[fc])
        if e2 < 0:
            continue
        for a in range(Np ** (dim - 1)):
            n1, n2 = face_node(dim, Np, l1, a), face_node(dim, Np, l2, a)
            s1 = 1.0 if l1 & 1 else -1.0
            s2 = 1.0 if l2 & 1 else -1.0
            np.testing.assert_allclose(m.face_node_nor[fc, a], s1 * m.node_adj[e1, n1, l1 >> 1], rtol=0, atol=1e-14)
            np.testing.assert_allclose(m.face_node_nor[fc, a], -s2 * m.node_adj[e2, n2, l2 >> 1], rtol=0, atol=1e-13)
