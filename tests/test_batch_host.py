"""Host side of the batch and serving forms (no GPU needed)."""
import ctypes as C

import numpy as np
import pytest

from prandtl_b200 import ensemble


def test_batch_config_defaults():
    from prandtl_b200 import _lib
    L = _lib.load()
    c = _lib.BatchConfig()
    L.prandtl_batch_config_default(C.byref(c))
    assert (c.precision, c.scheme, c.max_solves, c.steps_per_graph, c.use_graph) == (0, _lib.LSRK45, 4096, 4, 1)
    assert c.timeout_s == 120.0


def test_batch_create_validates_and_reports_missing_gpu():
    import torch
    from prandtl_b200 import _lib
    L = _lib.load()
    c = _lib.BatchConfig()
    L.prandtl_batch_config_default(C.byref(c))
    h = C.c_void_p()
    c.precision = 3
    assert L.prandtl_batch_create(C.byref(c), C.byref(h)) == _lib.PRANDTL_EUNSUPPORTED
    assert b"precision" in L.prandtl_batch_last_error(None)
    c.precision, c.scheme = 0, 7
    assert L.prandtl_batch_create(C.byref(c), C.byref(h)) == _lib.PRANDTL_EINVAL
    c.scheme = _lib.LSRK45
    if not torch.cuda.is_available():
        assert L.prandtl_batch_create(C.byref(c), C.byref(h)) == _lib.PRANDTL_ECUDA


def test_null_batch_and_server_calls_fail_cleanly():
    from prandtl_b200 import _lib
    L = _lib.load()
    assert L.prandtl_batch_destroy(None) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_advance(None, 1) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_sync(None) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_remove(None, 0) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_tune(None, 1) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_tune_in_steps(None) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_read_many(None, 0, None, None, 0) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_add_many(None, 0, None, None, None, 0, None, None) == _lib.PRANDTL_EINVAL
    assert L.prandtl_batch_kernel_launches(None) == 0
    assert L.prandtl_serve_destroy(None) == _lib.PRANDTL_EINVAL
    assert L.prandtl_serve_create(None, 1, None) == _lib.PRANDTL_EINVAL


def test_python_wrappers_validate_arguments():
    from prandtl_b200.batch import Batch
    with pytest.raises(ValueError):
        Batch("fp16")
    with pytest.raises(ValueError):
        Batch("fp32", "RK4")


def test_tgv_ensemble_draws_the_stated_distributions():
    ens = ensemble.tgv_ensemble(512)
    ns = np.array([m.n for m in ens])
    orders = np.array([m.order for m in ens])
    mach = np.array([m.mach for m in ens])
    re = np.array([m.re for m in ens])
    assert ns.min() >= 4 and ns.max() <= 16 and len(set(ns)) == 13
    assert set(orders) == {2, 3, 4, 5}
    assert mach.min() >= 0.05 and mach.max() <= 0.3
    assert re.min() >= 100 and re.max() <= 3200
    # log-uniform: the median is near the geometric mean of the bounds
    assert abs(np.log(np.median(re)) - 0.5 * np.log(100 * 3200)) < 0.35
    assert ensemble.tgv_ensemble(512)[17] == ens[17]          # seeded
    dofs = sum(m.dofs() for m in ens)
    assert 2.5e8 < dofs < 5.5e8                               # about 0.39 G DOF in total


def test_serving_stream_mix_and_arrivals():
    reqs = ensemble.serving_stream(2000, rate=10.0)
    kinds = [m.kind for m in reqs]
    assert 0.4 < kinds.count("tgv") / len(kinds) < 0.6
    t = np.array([m.arrival for m in reqs])
    assert np.all(np.diff(t) > 0)
    assert abs(np.mean(np.diff(t)) - 0.1) < 0.01               # Poisson, rate 10/s
    for m in reqs[:200]:
        assert 50 <= m.nsteps <= 500
        if m.kind == "tgv":
            assert 8 <= m.n <= 24 and m.order in (2, 3)
        else:
            assert 16 <= m.n <= 128 and m.order in (3, 4)


def test_fixed_dt_uses_the_initial_max_speed():
    m = ensemble.Member("tgv", 2, 3, mach=0.1)
    mesh = m.mesh()
    u0 = m.initial_state(mesh)
    lam = ensemble.max_char_speed(u0, 3)
    assert lam == pytest.approx(1 + np.sqrt(1 / 0.01), rel=0.05)   # |V| <= 1, c = 1/M
    assert ensemble.fixed_dt(mesh, u0, 0.5) == pytest.approx(0.5 * mesh.hmin / (lam * 16))
