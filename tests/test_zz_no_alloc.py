"""prandtl_rhs_noalloc: the RHS entry point for callers that cannot allocate.

Some callers cannot call cudaMalloc (they run inside another framework's
memory pool, or must keep a fixed device footprint).  This entry point takes
the mesh, state and output already in device memory and keeps its own scratch
in one fixed-size device array of the library.  The test calls it through the
C ABI twice in a row and checks each result against prandtl_rhs and against
the CPU oracle on the same input, within the parity tolerance used for the RHS
(1e-12 normalised), that the second call leaves the free device memory
unchanged, that a mesh too large for the fixed scratch is rejected before any
device work, and that the device-side mesh check rejects a mesh with a missing
face, a duplicated face or a non-positive det J (each a host-side fault in the
input arrays, which the check turns into PRANDTL_EUNSUPPORTED without running
the RHS kernels).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import normalized_error

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _device_desc(torch, mesh, keep):
    from prandtl_b200 import _lib
    dev = "cuda"
    arrs = [torch.from_numpy(np.ascontiguousarray(mesh.elem_adj).reshape(-1)).to(dev),
            torch.from_numpy(np.ascontiguousarray(mesh.elem_detj)).to(dev),
            torch.from_numpy(np.ascontiguousarray(mesh.face_elems, dtype=np.int32).reshape(-1)).to(dev),
            torch.from_numpy(np.ascontiguousarray(mesh.face_nor).reshape(-1)).to(dev)]
    keep.extend(arrs)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    return _lib.MeshDesc(mesh.dim, mesh.order, mesh.num_elements, mesh.num_faces,
                         C.cast(arrs[0].data_ptr(), dp), C.cast(arrs[1].data_ptr(), dp),
                         C.cast(arrs[2].data_ptr(), ip), C.cast(arrs[3].data_ptr(), dp))


def _config(L, **kw):
    from prandtl_b200 import _lib
    cfg = _lib.Config()
    L.prandtl_config_default(C.byref(cfg))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


CASES = [
    ("ns3d", 3, 3, 3, dict(parabolic=1, mu=1.0 / 1600.0, Pr=0.71)),
    ("euler2d_blend", 2, 6, 3, dict(blending=1, alpha_max=0.5)),
    ("ns2d_fixed", 2, 4, 4, dict(parabolic=1, mu=0.01, quirks=1)),
]


@pytest.mark.parametrize("name,dim,n,order,kw", CASES, ids=[c[0] for c in CASES])
def test_noalloc_rhs_matches_prandtl_rhs_on_two_calls(name, dim, n, order, kw, oracle_mod):
    torch = pytest.importorskip("torch")
    from prandtl_b200 import _lib, cases
    from prandtl_b200.mesh import periodic_box
    from prandtl_b200.operator import DGSEMOperator
    L = _lib.load()
    mesh = periodic_box(dim, n, order, 0.0, 1.0, affine=np.eye(dim) + 0.1 * np.ones((dim, dim)))
    u = cases.perturbed(mesh, cases.free_stream(mesh, rho=1.1), amp=0.3, seed=n)
    op_kw = {k: v for k, v in kw.items() if k != "quirks"}
    op_kw = {**op_kw, "parabolic": bool(op_kw.get("parabolic", 0)), "blending": bool(op_kw.get("blending", 0))}
    op = DGSEMOperator(mesh, quirks="fixed" if kw.get("quirks") else "reference", **op_kw)
    ref = np.empty_like(u)
    op.Mult(u, ref)
    okw = {k: v for k, v in kw.items()}
    okw.setdefault("quirks", 0)
    orc = oracle_mod.Oracle(mesh, **okw).rhs(u)["dudt"]

    keep = []
    desc = _device_desc(torch, mesh, keep)
    cfg = _config(L, **kw)
    ut = torch.from_numpy(u).cuda()
    out = torch.empty_like(ut)
    stream = torch.cuda.current_stream()
    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = L.prandtl_rhs_noalloc(C.byref(desc), C.byref(cfg), C.c_void_p(ut.data_ptr()),
                                   C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == _lib.PRANDTL_OK
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:   # the first call may load the module that holds the scratch array
            assert free_after == free_before
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        err = normalized_error(got, ref, mesh.num_fields)
        assert err <= TOL, f"call {call}: {err:.3e}"
        err_o = normalized_error(got, orc, mesh.num_fields)
        assert err_o <= TOL, f"call {call} vs oracle: {err_o:.3e}"


def test_noalloc_rejects_meshes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    from prandtl_b200 import _lib
    L = _lib.load()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    p = dummy.data_ptr()
    # 3D N=5 with 100k elements needs far more than the fixed scratch
    desc = _lib.MeshDesc(3, 5, 100000, 300000, C.cast(p, dp), C.cast(p, dp), C.cast(p, ip), C.cast(p, dp))
    cfg = _config(L, parabolic=1)
    rc = L.prandtl_rhs_noalloc(C.byref(desc), C.byref(cfg), C.c_void_p(p), C.c_void_p(p), None)
    assert rc == _lib.PRANDTL_ETOOLARGE
    assert b"scratch" in L.prandtl_last_error(None)


def _broken(mesh, how):
    """A copy of a periodic mesh with one face dropped or listed twice, or one
    element's det J negated (the arrays stay in range, so the check reads only
    valid memory)."""
    import copy
    m = copy.copy(mesh)
    faces = np.ascontiguousarray(mesh.face_elems, dtype=np.int32).copy()
    nor = np.ascontiguousarray(mesh.face_nor).copy()
    detj = np.ascontiguousarray(mesh.elem_detj).copy()
    if how == "missing":
        faces, nor = faces[1:], nor[1:]
    elif how == "duplicated":
        faces = np.concatenate([faces, faces[:1]])
        nor = np.concatenate([nor, nor[:1]])
    elif how == "detj":
        detj[3] = -detj[3]
    m.face_elems, m.face_nor, m.elem_detj = faces, nor, detj
    return m


@pytest.mark.parametrize("how", ["missing", "duplicated", "detj"])
def test_noalloc_device_mesh_check_rejects_bad_meshes(how):
    torch = pytest.importorskip("torch")
    from prandtl_b200 import _lib, cases
    from prandtl_b200.mesh import periodic_box
    L = _lib.load()
    mesh = periodic_box(3, 3, 2, 0.0, 1.0)
    u = torch.from_numpy(cases.free_stream(mesh)).cuda()
    out = torch.full_like(u, 7.0)
    keep = []
    desc = _device_desc(torch, _broken(mesh, how), keep)
    cfg = _config(L, parabolic=1, timeout_s=30.0)
    torch.cuda.synchronize()
    rc = L.prandtl_rhs_noalloc(C.byref(desc), C.byref(cfg), C.c_void_p(u.data_ptr()),
                               C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.PRANDTL_EUNSUPPORTED
    assert b"mesh invalid" in L.prandtl_last_error(None)
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())   # no RHS kernel ran
