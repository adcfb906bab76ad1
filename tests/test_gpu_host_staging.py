"""Host-pointer transfers of the one-operator path (marked gpu).

States above 4 MB cross between pageable host memory and the device through
a pinned ring of 8 MB chunks filled and emptied by host threads while the DMA
engine moves the neighbouring chunk.  These tests check that the staged
transfers deliver exactly the device-pointer results: Mult and Step with
numpy arrays against the same calls on torch CUDA tensors, for states of one
partial chunk, of two chunks, and of more chunks than the ring has slots
(slots reused within one transfer), twice in a row on one handle.
"""
import numpy as np
import pytest

from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

pytestmark = pytest.mark.gpu

NS = dict(parabolic=True, mu=1 / 1600, Pr=0.71, quirks="fixed")


@pytest.mark.parametrize("n", [10, 16, 24])   # 2.6, 10.5 and 35.4 MB states at N=3
def test_host_transfers_match_device_pointers(n):
    import torch
    from prandtl_b200.operator import DGSEMOperator
    mesh = periodic_box(3, n, 3, 0.0, 2 * np.pi)
    u0 = cases.taylor_green(mesh)
    op = DGSEMOperator(mesh, **NS)
    ud = torch.from_numpy(u0).cuda()
    dd = torch.empty_like(ud)
    op.Mult(ud, dd)
    op.synchronize()
    ref = dd.cpu().numpy()
    for _ in range(2):
        dh = np.full_like(u0, np.nan)
        op.Mult(u0, dh)
        assert np.array_equal(dh, ref)
    uh = u0.copy()
    op.Step(uh, 1e-3, scheme="LSRK45", nsteps=3)
    op.Step(ud, 1e-3, scheme="LSRK45", nsteps=3)
    op.synchronize()
    assert np.array_equal(uh, ud.cpu().numpy())
    op.close()
