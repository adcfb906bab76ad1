"""Resume through checkpoint files on the GPU path (marked gpu): stepping
N steps equals stepping k, saving, loading and stepping N - k, bit for bit."""
import numpy as np
import pytest

from prandtl_b200 import cases
from prandtl_b200.checkpoint import load_checkpoint, save_checkpoint
from prandtl_b200.mesh import periodic_box

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_resume_is_bit_identical(tmp_path, precision):
    from prandtl_b200.operator import DGSEMOperator
    mesh = periodic_box(3, 3, 3, 0.0, 2 * np.pi)
    u0 = cases.taylor_green(mesh)
    op = DGSEMOperator(mesh, parabolic=True, mu=1 / 1600, Pr=0.71, quirks="fixed", precision=precision)
    d = np.empty_like(u0)
    op.Mult(u0, d)
    dt = op.cfl_dt(0.1)
    full = u0.copy()
    op.Step(full, dt, scheme="LSRK45", nsteps=6)
    half = u0.copy()
    op.Step(half, dt, scheme="LSRK45", nsteps=4)
    save_checkpoint(tmp_path, 4, 4 * dt, mesh, half)
    u, t = load_checkpoint(tmp_path, 4, mesh)
    assert t == 4 * dt
    op.Step(u, dt, scheme="LSRK45", nsteps=2)
    op.close()
    assert np.array_equal(u, full)
