"""Write the small mesh files the mesh-ingestion tests read.

These are generated here (they are not the reference's mesh files): an MFEM
v1.0 periodic box with L2_T1 corner nodes (MFEM's periodic form), and Gmsh 2.2
ASCII boxes with physical groups whose elements list their vertices from
random starting corners (so the reader must re-orient them).

    python tests/golden/make_meshes.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "meshes")

QUAD_LEX = [0, 1, 3, 2]                 # lexicographic corner -> vertex slot
HEX_LEX = [0, 1, 3, 2, 4, 5, 7, 6]


def _grid(dim, n, lo, hi, shear):
    axes = [np.linspace(lo[d], hi[d], n[d] + 1) for d in range(dim)]
    pts = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)   # [i][j](k)[dim]
    return pts @ np.asarray(shear).T


def write_mfem_periodic_2d(path, n=(4, 3), lo=(0.0, 0.0), hi=(1.0, 1.0), shear=np.eye(2)):
    """Doubly periodic quad box: vertex ids identified across the box, corner
    coordinates per element in a nodes section (L2_T1_2D_P1, byVDIM)."""
    nx, ny = n
    X = _grid(2, n, lo, hi, shear)
    vid = lambda i, j: (i % nx) + nx * (j % ny)
    lines = ["MFEM mesh v1.0", "", "dimension", "2", "", "elements", str(nx * ny)]
    nodes = []
    for j in range(ny):
        for i in range(nx):
            lines.append(f"1 3 {vid(i, j)} {vid(i + 1, j)} {vid(i + 1, j + 1)} {vid(i, j + 1)}")
            for (a, b) in ((0, 0), (1, 0), (0, 1), (1, 1)):
                x = X[i + a, j + b]
                nodes.append(f"{x[0]:.17g} {x[1]:.17g}")
            nodes.append("")
    lines += ["", "boundary", "0", "", "vertices", str(nx * ny), "", "nodes", "FiniteElementSpace",
              "FiniteElementCollection: L2_T1_2D_P1", "VDim: 2", "Ordering: 1", ""] + nodes
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _proper_frames(dim):
    """Signed axis permutations with determinant +1, as (perm, flips)."""
    import itertools
    out = []
    for p in itertools.permutations(range(dim)):
        sign = np.linalg.det(np.eye(dim)[list(p)])
        for f in range(1 << dim):
            if sign * (-1) ** bin(f).count("1") > 0:
                out.append((p, f))
    return out


def _old_corner(frame, dim, b):
    p, f = frame
    return sum(((((b >> r) & 1) ^ ((f >> r) & 1)) << p[r]) for r in range(dim))


def write_gmsh_box(path, dim, n, lo, hi, shear=None, names=None, seed=0, warp=None):
    """Box of quads / hexes with one physical group per side (names[2*d+s]) and
    elements listed from a random proper rotation of their corners.  `warp`
    (a function of the grid points [..., dim], returning moved points) makes
    the elements non-affine."""
    rng = np.random.default_rng(seed)
    n = tuple(n)
    shear = np.eye(dim) if shear is None else np.asarray(shear)
    X = _grid(dim, n, lo, hi, shear)
    if warp is not None:
        X = warp(X)
    shape = tuple(v + 1 for v in n)
    nid = lambda idx: int(np.ravel_multi_index(idx, shape, order="F")) + 1
    names = names or [f"side{k}" for k in range(2 * dim)]
    frames = _proper_frames(dim)
    lex = QUAD_LEX if dim == 2 else HEX_LEX
    els = []
    for cell in np.ndindex(*n[::-1]):
        cell = cell[::-1]   # x fastest
        corners = [nid(tuple(cell[r] + ((b >> r) & 1) for r in range(dim))) for b in range(1 << dim)]
        fr = frames[rng.integers(len(frames))]
        listed = [corners[_old_corner(fr, dim, b)] for b in range(1 << dim)]
        slots = [0] * (1 << dim)
        for b in range(1 << dim):
            slots[lex[b]] = listed[b]
        els.append((3 if dim == 2 else 5, 2 * dim + 1, slots))
    for d in range(dim):
        for s in range(2):
            others = [r for r in range(dim) if r != d]
            for face in np.ndindex(*[n[r] for r in others][::-1]):
                face = face[::-1]
                corner = [0] * dim
                fc = []
                for b in range(1 << (dim - 1)):
                    for k, r in enumerate(others):
                        corner[r] = face[k] + ((b >> k) & 1)
                    corner[d] = s * n[d]
                    fc.append(nid(tuple(corner)))
                if dim == 3:
                    fc = [fc[0], fc[1], fc[3], fc[2]]
                els.append((1 if dim == 2 else 3, 2 * d + s + 1, fc))
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(2 * dim + 1)]
    for k, nm in enumerate(names):
        lines.append(f'{dim - 1} {k + 1} "{nm}"')
    lines.append(f'{dim} {2 * dim + 1} "fluid"')
    lines += ["$EndPhysicalNames", "$Nodes", str(int(np.prod(shape)))]
    for k, idx in enumerate(np.ndindex(*shape[::-1])):
        x = X[idx[::-1]]
        z = x[2] if dim == 3 else 0.0
        lines.append(f"{k + 1} {x[0]:.17g} {x[1]:.17g} {z:.17g}")
    lines += ["$EndNodes", "$Elements", str(len(els))]
    for k, (t, tag, v) in enumerate(els):
        lines.append(f"{k + 1} {t} 2 {tag} {tag} " + " ".join(map(str, v)))
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


SHEAR2 = np.array([[1.0, 0.2], [0.0, 1.1]])
SHEAR3 = np.array([[1.0, 0.1, 0.0], [0.0, 1.05, 0.15], [0.05, 0.0, 0.95]])


def main():
    os.makedirs(OUT, exist_ok=True)
    write_mfem_periodic_2d(os.path.join(OUT, "periodic_4x3.mesh"), (4, 3), (0.0, 0.0), (2.0, 1.5), SHEAR2)
    write_gmsh_box(os.path.join(OUT, "cavity_6x5.msh"), 2, (6, 5), (0.0, 0.0), (1.0, 1.0), SHEAR2,
                   ["left", "right", "bottom", "lid"], seed=1)
    write_gmsh_box(os.path.join(OUT, "channel_4x3x2.msh"), 3, (4, 3, 2), (0.0, 0.0, 0.0), (2.0, 1.0, 1.0), SHEAR3,
                   ["inlet", "outlet", "south", "north", "bottom", "top"], seed=2)
    # non-affine elements: a channel over a bump (trapezoids over the bump) and a
    # smoothly warped box of hexahedra
    def bump(X):
        x, y = X[..., 0], X[..., 1]
        floor = 0.12 * np.sin(np.pi * np.clip(x - 0.5, 0.0, 1.0)) ** 2
        return np.stack([x, floor + (1.0 - floor) * y], axis=-1)

    def wobble(X):
        x, y, z = X[..., 0], X[..., 1], X[..., 2]
        return np.stack([x + 0.04 * np.sin(np.pi * y) * np.sin(np.pi * z),
                         y + 0.05 * np.sin(np.pi * x / 2) * np.sin(np.pi * z),
                         z + 0.03 * np.sin(np.pi * x / 2) * np.sin(np.pi * y)], axis=-1)
    write_gmsh_box(os.path.join(OUT, "bump_8x4.msh"), 2, (8, 4), (0.0, 0.0), (2.0, 1.0), None,
                   ["inlet", "outlet", "floor", "top"], seed=3, warp=bump)
    write_gmsh_box(os.path.join(OUT, "warped_3x3x2.msh"), 3, (3, 3, 2), (0.0, 0.0, 0.0), (2.0, 1.0, 1.0), None,
                   ["inlet", "outlet", "south", "north", "bottom", "top"], seed=4, warp=wobble)
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
