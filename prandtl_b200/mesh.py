"""Periodic hexahedral / quadrilateral meshes in the descriptor form the C-ABI takes.

The reference reads its meshes through MFEM (``Simulation.cpp:271-336``) and the
DGSEM kernels only ever see, per element, the affine Jacobian's adjugate and
determinant (``ElementTransformation::AdjugateJacobian`` / ``Weight``), and per
interior face the two neighbouring elements plus MFEM's ``CalcOrtho`` scaled
normal (outward from ``Elem1``).  This module builds exactly that for a
periodic box of ``n[0] x ... x n[dim-1]`` elements, optionally sheared by a
global affine map (every element stays a parallelogram / parallelepiped).

Element order is lexicographic (x fastest).  Which element of a face is
``Elem1`` follows MFEM's face generation: elements are visited in order and
each element's local faces in MFEM's local order; the first visitor owns the
face.  For n >= 2 that is the lower element index; for n == 1 the face joins an
element to itself and the first local face in MFEM's order is Elem1's.

Local faces are numbered ``lf = 2*dir + side`` (side 0: xi_dir = 0).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# MFEM's local face order as (dir, side): Geometry::SQUARE faces 0..3 are
# y=0, x=1, y=1, x=0; Geometry::CUBE faces 0..5 are z=0, y=0, x=1, y=1, x=0, z=1.
_MFEM_FACE_ORDER = {
    2: [(1, 0), (0, 1), (1, 1), (0, 0)],
    3: [(2, 0), (1, 0), (0, 1), (1, 1), (0, 0), (2, 1)],
}


def gauss_lobatto(order: int):
    """Gauss-Lobatto nodes and weights on [0, 1] (long-double Newton on P'_N)."""
    N = order
    Np = N + 1
    if N < 1:
        raise ValueError("order must be >= 1")
    xs = np.empty(Np, dtype=np.longdouble)
    for i in range(Np):
        xi = -np.cos(np.longdouble(np.pi) * i / N)
        if 0 < i < N:
            for _ in range(100):
                p0, p1, dp0, dp1 = np.longdouble(1), xi, np.longdouble(0), np.longdouble(1)
                for k in range(1, N):
                    p2 = ((2 * k + 1) * xi * p1 - k * p0) / (k + 1)
                    dp2 = dp0 + (2 * k + 1) * p1
                    p0, p1, dp0, dp1 = p1, p2, dp1, dp2
                f = (1 - xi * xi) * dp1
                fp = -np.longdouble(N * (N + 1)) * p1
                dx = f / fp
                xi = xi - dx
                if abs(dx) < 1e-30:
                    break
        xs[i] = xi
    w = np.empty(Np, dtype=np.longdouble)
    for i in range(Np):
        p0, p1 = np.longdouble(1), xs[i]
        for k in range(1, N):
            p0, p1 = p1, ((2 * k + 1) * xs[i] * p1 - k * p0) / (k + 1)
        w[i] = 2 / (np.longdouble(N * (N + 1)) * p1 * p1)
    x = np.array((xs + 1) * 0.5, dtype=np.float64)
    x[0], x[-1] = 0.0, 1.0
    return x, np.array(w * 0.5, dtype=np.float64)


def _adjugate(J: np.ndarray) -> np.ndarray:
    """Explicit 2x2 / 3x3 adjugate (as MFEM's CalcAdjugate)."""
    d = J.shape[0]
    if d == 2:
        return np.array([[J[1, 1], -J[0, 1]], [-J[1, 0], J[0, 0]]])
    a = np.empty((3, 3))
    a[0, 0] = J[1, 1] * J[2, 2] - J[1, 2] * J[2, 1]
    a[0, 1] = J[0, 2] * J[2, 1] - J[0, 1] * J[2, 2]
    a[0, 2] = J[0, 1] * J[1, 2] - J[0, 2] * J[1, 1]
    a[1, 0] = J[1, 2] * J[2, 0] - J[1, 0] * J[2, 2]
    a[1, 1] = J[0, 0] * J[2, 2] - J[0, 2] * J[2, 0]
    a[1, 2] = J[0, 2] * J[1, 0] - J[0, 0] * J[1, 2]
    a[2, 0] = J[1, 0] * J[2, 1] - J[1, 1] * J[2, 0]
    a[2, 1] = J[0, 1] * J[2, 0] - J[0, 0] * J[2, 1]
    a[2, 2] = J[0, 0] * J[1, 1] - J[0, 1] * J[1, 0]
    return a


def _det(J: np.ndarray) -> float:
    if J.shape[0] == 2:
        return float(J[0, 0] * J[1, 1] - J[0, 1] * J[1, 0])
    return float(J[0, 0] * (J[1, 1] * J[2, 2] - J[1, 2] * J[2, 1])
                 - J[0, 1] * (J[1, 0] * J[2, 2] - J[1, 2] * J[2, 0])
                 + J[0, 2] * (J[1, 0] * J[2, 1] - J[1, 1] * J[2, 0]))


@dataclass
class Mesh:
    """Descriptor arrays for ``prandtl_mesh_desc`` plus node coordinates."""

    dim: int
    order: int
    n: tuple
    elem_adj: np.ndarray      # (E, dim, dim) float64
    elem_detj: np.ndarray     # (E,) float64
    face_elems: np.ndarray    # (F, 4) int32: elem1, lface1, elem2, lface2
    face_nor: np.ndarray      # (F, dim) float64
    coords: np.ndarray        # (dim, E*Np^dim) physical node coordinates
    hmin: float               # min element size (MFEM GetElementSize(e, 1))
    nodes_1d: np.ndarray = field(default=None)
    weights_1d: np.ndarray = field(default=None)
    face_attr: np.ndarray = field(default=None)   # (F,) boundary attribute per face (read meshes)
    elem_attr: np.ndarray = field(default=None)   # (E,) element attribute (read meshes)
    # non-affine (multilinear) elements: the transformation at every node and the
    # scaled normal at every face node (None for affine meshes, whose elem_adj /
    # elem_detj / face_nor hold for every node)
    node_adj: np.ndarray = field(default=None)        # (E, Np^dim, dim, dim)
    node_detj: np.ndarray = field(default=None)       # (E, Np^dim)
    face_node_nor: np.ndarray = field(default=None)   # (F, Np^(dim-1), dim), elem1's face node order

    @property
    def affine(self) -> bool:
        return self.node_adj is None

    @property
    def Np(self) -> int:
        return self.order + 1

    @property
    def nodes_per_elem(self) -> int:
        return self.Np ** self.dim

    @property
    def num_elements(self) -> int:
        return int(self.elem_detj.shape[0])

    @property
    def num_faces(self) -> int:
        return int(self.face_elems.shape[0])

    @property
    def ndof(self) -> int:
        """Nodes per field (MFEM's scalar dof count)."""
        return self.num_elements * self.nodes_per_elem

    @property
    def num_fields(self) -> int:
        return self.dim + 2

    def node_weights(self) -> np.ndarray:
        """Quadrature weight w_i w_j (w_k) * |J| per node, shape (E*Np^dim,)."""
        w = self.weights_1d
        if self.dim == 2:
            wn = np.outer(w, w).reshape(-1)          # [j][i] -> node j*Np+i
        else:
            wn = np.einsum("k,j,i->kji", w, w, w).reshape(-1)
        detj = self.elem_detj[:, None] if self.node_detj is None else self.node_detj
        return (detj * wn[None, :]).reshape(-1)


def face_node(dim: int, Np: int, lf: int, a: int) -> int:
    """Element-local node of face node a on local face lf = 2*dir + side (face
    nodes lexicographic over the remaining directions, lower direction fastest)."""
    d, s = lf >> 1, lf & 1
    c = [0, 0, 0]
    c[d] = s * (Np - 1)
    if dim == 2:
        c[1 - d] = a
    else:
        t0 = 1 if d == 0 else 0
        t1 = 1 if d == 2 else 2
        c[t0], c[t1] = a % Np, a // Np
    return c[0] + Np * c[1] + Np * Np * c[2]


def multilinear_geometry(corners: np.ndarray, x1: np.ndarray):
    """Node coordinates, Jacobian adjugates and determinants of multilinear
    elements (MFEM's bilinear quadrilateral / trilinear hexahedron map) at the
    tensor Gauss-Lobatto nodes x1.

    corners: (E, 2^dim, dim), corner b at reference vertex (b & 1, b >> 1 & 1,
    b >> 2 & 1).  Returns coords (dim, E*Np^dim), adj (E, Np^dim, dim, dim),
    detj (E, Np^dim), with J[i][r] = dx_i / dxi_r."""
    E, nc, dim = corners.shape
    Np = len(x1)
    grids = np.meshgrid(*([x1] * dim), indexing="ij")
    ref = np.stack([g.transpose().reshape(-1) for g in grids], axis=1)   # (nd, dim), x fastest
    nd = ref.shape[0]
    bits = np.array([[(b >> r) & 1 for r in range(dim)] for b in range(nc)], dtype=np.float64)   # (nc, dim)
    # phi_b(xi) = prod_r (xi_r if bit else 1 - xi_r); dphi_b / dxi_r
    fac = np.where(bits[None, :, :] > 0, ref[:, None, :], 1.0 - ref[:, None, :])   # (nd, nc, dim)
    phi = fac.prod(axis=2)                                                       # (nd, nc)
    dphi = np.empty((nd, nc, dim))
    for r in range(dim):
        others = np.prod(np.delete(fac, r, axis=2), axis=2) if dim > 1 else 1.0
        dphi[:, :, r] = np.where(bits[None, :, r] > 0, 1.0, -1.0) * others
    X = np.einsum("kb,ebi->eki", phi, corners)            # (E, nd, dim)
    J = np.einsum("kbr,ebi->ekir", dphi, corners)         # (E, nd, dim, dim)
    adj = np.empty_like(J)
    detj = np.empty(J.shape[:2])
    for e in range(E):
        for k in range(nd):
            adj[e, k] = _adjugate(J[e, k])
            detj[e, k] = _det(J[e, k])
    coords = np.ascontiguousarray(X.transpose(2, 0, 1).reshape(dim, E * nd))
    return coords, adj, detj


def periodic_box(dim: int, n, order: int, lo=0.0, hi=1.0, affine=None, bcs=None, warp=None) -> Mesh:
    """Box mesh [lo, hi]^dim with n elements per direction, periodic unless
    ``bcs`` says otherwise.

    ``n`` may be an int or a per-direction tuple; ``lo``/``hi`` scalars or
    per-direction tuples.  ``affine`` (dim x dim) maps the box afterwards,
    x = affine @ X, keeping every element affine.  ``warp`` (a function of the
    box coordinates X, shape (dim, npts), returning displacements of the same
    shape; periodic in the periodic directions) moves every element corner to
    affine @ X + warp(X): the elements become multilinear (non-affine) and the
    mesh carries per-node geometry.  ``bcs`` (length 2*dim,
    entry 2*d + side for the side x_d = lo (0) or hi (1)) holds None for a
    periodic direction or the boundary-condition index of that side's
    boundary faces, listed as (elem, local face, -1, bc index).
    """
    if dim not in (2, 3):
        raise ValueError("dim must be 2 or 3")
    n = tuple([n] * dim) if np.isscalar(n) else tuple(int(v) for v in n)
    lo = np.broadcast_to(np.asarray(lo, dtype=np.float64), (dim,)).copy()
    hi = np.broadcast_to(np.asarray(hi, dtype=np.float64), (dim,)).copy()
    M = np.eye(dim) if affine is None else np.asarray(affine, dtype=np.float64)
    h = (hi - lo) / np.asarray(n, dtype=np.float64)
    E = int(np.prod(n))
    J = M @ np.diag(h)
    adj = _adjugate(J)
    detj = _det(J)
    elem_adj = np.broadcast_to(adj, (E, dim, dim)).copy()
    elem_detj = np.full(E, detj)

    # element index <-> cell coordinates (x fastest)
    idx = np.arange(E)
    cell = np.stack([(idx // int(np.prod(n[:d]))) % n[d] for d in range(dim)])   # (dim, E)
    strides = [int(np.prod(n[:d])) for d in range(dim)]
    order_pos = {fs: p for p, fs in enumerate(_MFEM_FACE_ORDER[dim])}

    bcs = [None] * (2 * dim) if bcs is None else list(bcs)
    if len(bcs) != 2 * dim or any((bcs[2 * d] is None) != (bcs[2 * d + 1] is None) for d in range(dim)):
        raise ValueError("bcs: 2*dim entries, both sides of a direction periodic (None) or both bounded")
    faces = []
    normals = []
    for d in range(dim):
        up = cell.copy()
        up[d] = (up[d] + 1) % n[d]
        e_up = sum(up[k] * strides[k] for k in range(dim))
        for e in range(E):
            eu = int(e_up[e])
            if bcs[2 * d] is not None:   # bounded direction: interior faces plus two boundary sides
                if cell[d, e] == 0:
                    faces.append((e, 2 * d + 0, -1, int(bcs[2 * d])))
                    normals.append(-adj[d])
                if cell[d, e] == n[d] - 1:
                    faces.append((e, 2 * d + 1, -1, int(bcs[2 * d + 1])))
                    normals.append(+adj[d])
                else:
                    faces.append((e, 2 * d + 1, eu, 2 * d + 0))
                    normals.append(+adj[d])
            elif n[d] >= 2:
                if e < eu:
                    faces.append((e, 2 * d + 1, eu, 2 * d + 0))
                    normals.append(+adj[d])
                else:
                    faces.append((eu, 2 * d + 0, e, 2 * d + 1))
                    normals.append(-adj[d])
            else:
                first_side = 0 if order_pos[(d, 0)] < order_pos[(d, 1)] else 1
                faces.append((e, 2 * d + first_side, e, 2 * d + 1 - first_side))
                normals.append(adj[d] if first_side == 1 else -adj[d])
    face_elems = np.asarray(faces, dtype=np.int32).reshape(-1, 4)
    face_nor = np.asarray(normals, dtype=np.float64).reshape(-1, dim)

    x1, w1 = gauss_lobatto(order)
    Np = order + 1
    # reference-cell node coordinates, lexicographic x fastest
    grids = np.meshgrid(*([x1] * dim), indexing="ij")   # grids[d][i0,i1,(i2)]
    ref = np.stack([g.transpose().reshape(-1) for g in grids])   # (dim, Np^dim)
    X = lo[:, None, None] + (cell[:, :, None] + ref[:, None, :]) * h[:, None, None]   # (dim,E,nd)
    coords = np.einsum("ab,bek->aek", M, X).reshape(dim, -1)
    # GetElementSize(e, 1): smallest singular value of J
    hmin = float(np.linalg.svd(J, compute_uv=False).min())
    mesh = Mesh(dim=dim, order=order, n=n, elem_adj=elem_adj, elem_detj=elem_detj,
                face_elems=face_elems, face_nor=face_nor, coords=coords, hmin=hmin,
                nodes_1d=x1, weights_1d=w1)
    if warp is not None:
        nc = 1 << dim
        bits = np.array([[(b >> r) & 1 for r in range(dim)] for b in range(nc)])   # (nc, dim)
        Xc = lo[None, None, :] + (cell.T[:, None, :] + bits[None, :, :]) * h[None, None, :]   # (E, nc, dim)
        flat = Xc.reshape(-1, dim).T
        corners = (M @ flat + np.asarray(warp(flat), dtype=np.float64)).T.reshape(E, nc, dim)
        set_multilinear(mesh, corners)
    return mesh


def set_multilinear(mesh: Mesh, corners: np.ndarray) -> None:
    """Give ``mesh`` the geometry of multilinear elements with these corners
    ((E, 2^dim, dim), corner b at reference vertex bits of b, in each element's
    local frame): node coordinates, per-node adjugates and determinants, the
    scaled normal at every face node (outward from elem1: +/- the adjugate row
    of the face direction at elem1's face node, which is MFEM's CalcOrtho of the
    face Jacobian), element values at the centre, and hmin as MFEM's
    GetElementSize(e, 1) (smallest singular value of J at the centre)."""
    dim, Np = mesh.dim, mesh.order + 1
    x1 = mesh.nodes_1d
    coords, adj, detj = multilinear_geometry(corners, x1)
    if not (detj > 0).all():
        raise ValueError("inverted element (det J <= 0 at a node)")
    _, cadj, cdet = multilinear_geometry(corners, np.array([0.5]))
    nfn = Np ** (dim - 1)
    F = mesh.num_faces
    fnn = np.empty((F, nfn, dim))
    for fc in range(F):
        e1, lf1 = int(mesh.face_elems[fc, 0]), int(mesh.face_elems[fc, 1])
        d, sgn = lf1 >> 1, (1.0 if lf1 & 1 else -1.0)
        for a in range(nfn):
            fnn[fc, a] = sgn * adj[e1, face_node(dim, Np, lf1, a), d]
    Jc = np.array([[[0.0] * dim] * dim] * corners.shape[0])
    # centre Jacobian from the centre adjugate: J = adj(adj) / det^(dim-2)
    for e in range(corners.shape[0]):
        Jc[e] = _adjugate(cadj[e, 0]) / (cdet[e, 0] ** (dim - 2))
    mesh.coords = coords
    mesh.node_adj = adj
    mesh.node_detj = detj
    mesh.face_node_nor = fnn
    mesh.elem_adj = np.ascontiguousarray(cadj[:, 0])
    mesh.elem_detj = np.ascontiguousarray(cdet[:, 0])
    mesh.face_nor = np.ascontiguousarray(fnn.mean(axis=1))
    mesh.hmin = float(min(np.linalg.svd(Jc[e], compute_uv=False).min() for e in range(corners.shape[0])))


def read_mesh(path: str, order: int, refine: int = 0, hilbert: bool = False, boundary_conditions=None) -> Mesh:
    """Read an MFEM v1.0 or Gmsh 2.2 ASCII mesh through the native reader
    (``prandtl_mesh_read``: quadrilaterals / hexahedra with aligned frames;
    non-affine elements come back multilinear, with per-node geometry).

    ``refine`` uniform refinements and ``hilbert`` element ordering follow the
    reference's ``ser_ref_levels`` and ``"mesh_ordering": "Hilbert"``.
    ``boundary_conditions`` maps a boundary attribute (int) or a Gmsh physical
    name to a BC index; boundary faces default to BC index attribute - 1.
    """
    import ctypes as C
    from . import _lib
    L = _lib.load()
    h = C.c_void_p()
    st = L.prandtl_mesh_read(str(path).encode(), int(order), int(refine), int(bool(hilbert)), C.byref(h))
    if st != _lib.PRANDTL_OK:
        raise _lib.PrandtlError(st, L.prandtl_mesh_last_error().decode(errors="replace"))
    try:
        dim_probe = _lib.MeshDesc()
        hmin = C.c_double()
        L.prandtl_mesh_describe(h, C.byref(dim_probe), C.byref(hmin))
        F = dim_probe.num_faces
        fattr = np.zeros(F, dtype=np.int32)
        L.prandtl_mesh_face_attributes(h, fattr.ctypes.data_as(C.POINTER(C.c_int)))
        if boundary_conditions:
            amax = int(fattr.max(initial=0))
            table = np.full(max(amax, 1), -1, dtype=np.int32)
            for a in range(1, amax + 1):
                table[a - 1] = a - 1
            for key, bc in boundary_conditions.items():
                a = key if isinstance(key, (int, np.integer)) else \
                    L.prandtl_mesh_attribute(h, dim_probe.dim - 1, str(key).encode())
                if a < 1:
                    raise KeyError(f"no boundary attribute named {key!r}")
                if a > amax:
                    continue
                table[a - 1] = int(bc)
            L.prandtl_mesh_set_boundary_conditions(h, table.ctypes.data_as(C.POINTER(C.c_int)), int(table.size))
        d = _lib.MeshDesc()
        L.prandtl_mesh_describe(h, C.byref(d), None)
        dim, E = d.dim, d.num_elements
        adj = np.ctypeslib.as_array(d.elem_adj, shape=(E * dim * dim,)).reshape(E, dim, dim).copy()
        detj = np.ctypeslib.as_array(d.elem_detj, shape=(E,)).copy()
        faces = np.ctypeslib.as_array(d.face_elems, shape=(F * 4,)).reshape(F, 4).copy()
        nor = np.ctypeslib.as_array(d.face_nor, shape=(F * dim,)).reshape(F, dim).copy()
        Np = order + 1
        coords = np.empty((dim, E * Np ** dim))
        L.prandtl_mesh_node_coords(h, coords.ctypes.data_as(C.POINTER(C.c_double)))
        eattr = np.empty(E, dtype=np.int32)
        L.prandtl_mesh_element_attributes(h, eattr.ctypes.data_as(C.POINTER(C.c_int)))
        node = None
        if d.node_adj:   # multilinear elements: the per-node arrays
            nd, nfn = Np ** dim, Np ** (dim - 1)
            node = (np.ctypeslib.as_array(d.node_adj, shape=(E * nd * dim * dim,)).reshape(E, nd, dim, dim).copy(),
                    np.ctypeslib.as_array(d.node_detj, shape=(E * nd,)).reshape(E, nd).copy(),
                    np.ctypeslib.as_array(d.face_node_nor, shape=(F * nfn * dim,)).reshape(F, nfn, dim).copy())
    finally:
        L.prandtl_mesh_destroy(h)
    x, w = gauss_lobatto(order)
    mesh = Mesh(dim=dim, order=order, n=(E,), elem_adj=adj, elem_detj=detj, face_elems=faces.astype(np.int32),
                face_nor=nor, coords=coords, hmin=float(hmin.value), nodes_1d=x, weights_1d=w,
                face_attr=fattr, elem_attr=eattr)
    if node is not None:
        mesh.node_adj, mesh.node_detj, mesh.face_node_nor = node
    return mesh
