"""C-ABI library: loads, exports every declared symbol, validates input without a GPU."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from prandtl_b200 import _lib, build
    if build.needs_build():
        build.build()
    return _lib.load()


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(prandtl_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported(lib):
    from prandtl_b200 import _lib
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    assert set(names) == set(_lib.EXPORTS)


def test_config_defaults(lib):
    from prandtl_b200 import _lib
    c = _lib.Config()
    lib.prandtl_config_default(C.byref(c))
    assert (c.gamma, c.Pr, c.mu, c.R_gas) == (1.4, 0.72, 0.02, 287.05)
    assert (c.alpha_max, c.alpha_min) == (0.5, 0.001)
    assert c.surface_dissipation == 1 and c.quirks == 0 and c.precision == 0


def test_cfl_dt(lib):
    assert lib.prandtl_cfl_dt(0.5, 0.3125, 2.0, 3) == pytest.approx(0.5 * 0.3125 / (2.0 * 16))


def _desc(mesh, keep):
    from prandtl_b200 import _lib
    dp = C.POINTER(C.c_double)
    keep += [np.ascontiguousarray(mesh.elem_adj), np.ascontiguousarray(mesh.elem_detj),
             np.ascontiguousarray(mesh.face_elems, dtype=np.int32), np.ascontiguousarray(mesh.face_nor)]
    return _lib.MeshDesc(mesh.dim, mesh.order, mesh.num_elements, mesh.num_faces,
                         keep[-4].ctypes.data_as(dp), keep[-3].ctypes.data_as(dp),
                         keep[-2].ctypes.data_as(C.POINTER(C.c_int)), keep[-1].ctypes.data_as(dp))


def test_create_validates_before_touching_the_device(lib):
    from prandtl_b200 import _lib
    from prandtl_b200.mesh import periodic_box
    keep = []
    cfg = _lib.Config()
    lib.prandtl_config_default(C.byref(cfg))
    h = C.c_void_p()
    assert lib.prandtl_create(None, C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EINVAL
    m = periodic_box(2, 2, 3)
    d = _desc(m, keep)
    d.order = 7
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    assert b"order" in lib.prandtl_last_error(None)
    d = _desc(m, keep)
    d.num_faces -= 1   # an element face without a neighbour
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    cfg.precision = 2
    d = _desc(m, keep)
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED


def test_create_without_gpu_reports_ecuda(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from prandtl_b200 import _lib
    from prandtl_b200.operator import DGSEMOperator
    from prandtl_b200.mesh import periodic_box
    with pytest.raises(_lib.PrandtlError) as ei:
        DGSEMOperator(periodic_box(2, 2, 3))
    assert ei.value.status == _lib.PRANDTL_ECUDA


def test_null_handle_calls_fail_cleanly(lib):
    from prandtl_b200 import _lib
    assert lib.prandtl_destroy(None) == _lib.PRANDTL_EINVAL
    assert lib.prandtl_rhs(None, None, None, 0.0, None, 0) == _lib.PRANDTL_EINVAL
    assert lib.prandtl_step(None, None, 0.0, 0.1, 0, 1, 0) == _lib.PRANDTL_EINVAL
    assert lib.prandtl_synchronize(None) == _lib.PRANDTL_EINVAL
    assert lib.prandtl_budgets(None, None, None, None, 0) == _lib.PRANDTL_EINVAL
    assert lib.prandtl_batch_budgets(None, 0, None) == _lib.PRANDTL_EINVAL
    assert lib.prandtl_recover_state(None, None, None, 0) == _lib.PRANDTL_EINVAL
    assert lib.prandtl_kernel_launches(None) == 0
    assert lib.prandtl_version().startswith(b"prandtl_b200")


def test_face_normals_must_match_the_metrics_in_fixed_navier_stokes(lib):
    """Fixed-mode NS takes face viscous terms from the adjugate rows; a mesh whose
    face normals disagree with them is rejected before any device work."""
    from prandtl_b200 import _lib
    from prandtl_b200.mesh import periodic_box
    keep = []
    cfg = _lib.Config()
    lib.prandtl_config_default(C.byref(cfg))
    cfg.parabolic, cfg.quirks = 1, 1
    m = periodic_box(3, 2, 2, 0.0, 1.0, affine=np.array([[1.0, 0.2, 0.0], [0.0, 1.1, 0.1], [0.05, 0.0, 0.9]]))
    h = C.c_void_p()
    m.face_nor = np.array(m.face_nor, copy=True)
    m.face_nor[3, 1] += 1e-3
    d = _desc(m, keep)
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    assert b"adjugate" in lib.prandtl_last_error(None)
    cfg.quirks = 0   # reference mode evaluates viscous fluxes from gradients: no such requirement
    st = lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h))
    assert st in (_lib.PRANDTL_ECUDA, _lib.PRANDTL_OK)
    if st == _lib.PRANDTL_OK:
        lib.prandtl_destroy(h)



def test_boundary_tables_validated_before_touching_the_device(lib):
    """Boundary faces {e1, l1, -1, bc}: a bad BC index, type or datum is EINVAL;
    Navier-Stokes with a condition that has no viscous treatment is
    EUNSUPPORTED; all before device work."""
    from prandtl_b200 import _lib
    from prandtl_b200.mesh import periodic_box
    from prandtl_b200.operator import make_config
    keep = []
    h = C.c_void_p()
    m = periodic_box(2, 2, 2, 0.0, 1.0, bcs=[0, 0, None, None])
    assert (m.face_elems[:, 2] == -1).sum() == 4
    d = _desc(m, keep)
    cfg = make_config()    # no BC table: the faces name BC 0 of none
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EINVAL
    assert b"boundary condition" in lib.prandtl_last_error(None)
    cfg = make_config(bcs=[("outflow",)])
    cfg._bcs[0].type = 42
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EINVAL
    assert b"unknown type" in lib.prandtl_last_error(None)
    cfg = make_config(bcs=[("state", [0.0, 0.1, 0.0, 2.5])])
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EINVAL
    for kind in ("slip_wall", "symmetry"):   # no viscous treatment in the reference
        cfg = make_config(bcs=[(kind,)], parabolic=True)
        assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
        assert b"viscous" in lib.prandtl_last_error(None)
    cfg = make_config(bcs=[("riemann", [1.2, 0.3, 0.0, 1.5])], parabolic=True, quirks="reference")
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    cfg = make_config(bcs=[("noslip_isothermal", dict(wall_T=0.0))], parabolic=True)
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EINVAL
    for kw in (dict(bcs=[("outflow",)]), dict(bcs=[("outflow",)], parabolic=True),
               dict(bcs=[("noslip_adiabatic", dict(wall_vel=[1.0, 0.0]))], parabolic=True),
               dict(bcs=[("riemann", [1.2, 0.3, 0.0, 1.5])], parabolic=True, quirks="fixed")):
        cfg = make_config(**kw)
        st = lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h))
        assert st in (_lib.PRANDTL_ECUDA, _lib.PRANDTL_OK), kw
        if st == _lib.PRANDTL_OK:
            lib.prandtl_destroy(h)


def test_axisymmetric_configuration_checked_before_the_device(lib):
    """The axisymmetric form is 2D Euler with node coordinates; the axis
    condition needs it; the no-alloc entry point leaves it to prandtl_create.
    All checked before device work."""
    from prandtl_b200 import _lib
    from prandtl_b200.mesh import periodic_box
    from prandtl_b200.operator import make_config
    keep = []
    h = C.c_void_p()
    m = periodic_box(2, (3, 2), 2, (0.0, 0.0), (1.0, 1.0), bcs=[0, 0, 1, 0])
    d = _desc(m, keep)
    bcs = [("outflow",), ("axis",)]
    cfg = make_config(bcs=bcs)   # axis without the axisymmetric form
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    assert b"axisymmetric" in lib.prandtl_last_error(None)
    cfg = make_config(bcs=bcs, axisymmetric=True)   # no node coordinates
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EINVAL
    cfg = make_config(bcs=bcs, axisymmetric=True, node_coords=m.coords, parabolic=True)
    assert lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    m3 = periodic_box(3, 2, 2)
    d3 = _desc(m3, keep)
    cfg = make_config(axisymmetric=True, node_coords=m3.coords)
    assert lib.prandtl_create(C.byref(d3), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    cfg = make_config(bcs=bcs, axisymmetric=True, node_coords=m.coords)
    st = lib.prandtl_create(C.byref(d), C.byref(cfg), C.byref(h))
    assert st in (_lib.PRANDTL_ECUDA, _lib.PRANDTL_OK)
    if st == _lib.PRANDTL_OK:
        lib.prandtl_destroy(h)
    u = np.zeros(m.num_fields * m.ndof)
    assert lib.prandtl_rhs_noalloc(C.byref(d), C.byref(cfg), u.ctypes.data, u.ctypes.data, None) == \
        _lib.PRANDTL_EUNSUPPORTED


def test_non_affine_descriptor_checked_before_the_device(lib):
    """Per-node geometry: all three arrays or none, positive det J, FP64 or
    FP32-bulk Euler, and in fixed Navier-Stokes the face-node normals must be
    the adjugate rows."""
    import sys
    from prandtl_b200 import _lib
    from prandtl_b200.mesh import periodic_box
    from prandtl_b200.operator import MeshArrays, make_config
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_golden
    def mesh():   # MeshArrays shares the mesh's arrays: a fresh mesh per altered copy
        return periodic_box(2, 3, 2, warp=make_golden.warp_field(2, 0.06))
    arr = MeshArrays(mesh())
    h = C.c_void_p()
    st = lib.prandtl_create(C.byref(arr.desc), C.byref(make_config(precision="fp32", parabolic=True)), C.byref(h))
    assert st == _lib.PRANDTL_EUNSUPPORTED
    assert b"FP64" in lib.prandtl_last_error(None)
    part = MeshArrays(mesh())
    part.desc.face_node_nor = None
    assert lib.prandtl_create(C.byref(part.desc), C.byref(make_config()), C.byref(h)) == _lib.PRANDTL_EINVAL
    bad = MeshArrays(mesh())
    bad.node[1][3, 2] = -1.0
    assert lib.prandtl_create(C.byref(bad.desc), C.byref(make_config()), C.byref(h)) == _lib.PRANDTL_EINVAL
    skew = MeshArrays(mesh())
    skew.node[2][4, 1, 0] += 1e-3
    cfg = make_config(parabolic=True, quirks="fixed")
    assert lib.prandtl_create(C.byref(skew.desc), C.byref(cfg), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    # a valid descriptor gets as far as the device
    st = lib.prandtl_create(C.byref(arr.desc), C.byref(make_config(parabolic=True, quirks="fixed")), C.byref(h))
    assert st in (_lib.PRANDTL_ECUDA, _lib.PRANDTL_OK)
    if st == _lib.PRANDTL_OK:
        lib.prandtl_destroy(h)
