"""Device unit tests of the point-wise routines the kernels share (marked gpu).

rcp(x) (dgsem_device.cuh): the hardware reciprocal estimate refined by two
Newton-Raphson steps in FP64 (Markstein's method), the estimate alone in FP32.
It replaces the reference's divisions, so it must stay within one ulp of
CUDA's correctly rounded 1/x: swept over x in [1e-6, 1e6].

log_mean(x, y) (BasicOperations.cpp:6-12): the logarithmic mean on its series
branch (f = (y-x)/(y+x), u = f^2 below 1e-4 in FP64, below 0.04 in the
FP32-bulk form) and its logarithm branch, against a long-double evaluation of
(y - x) / (ln y - ln x), densely across both switches.  The reference's own
series, (x+y) 52.5/(105 + u(35 + u(21 + 15u))), is checked beside it on the
host: both agree with the exact mean to FP64 rounding.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def dm(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("dm") / "libdevice_math.so")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-Xcompiler", "-fPIC", "-shared", os.path.join(ROOT, "tests", "cpp", "device_math.cu"),
                    "-o", out], check=True)
    L = C.CDLL(out)
    for name, T in (("dm_rcp64", C.c_double), ("dm_rcp32", C.c_float)):
        fn = getattr(L, name)
        fn.argtypes = [C.POINTER(T)] * 3 + [C.c_int]
        fn.restype = C.c_int
    for name, T in (("dm_log_mean64", C.c_double), ("dm_log_mean32", C.c_float)):
        fn = getattr(L, name)
        fn.argtypes = [C.POINTER(T)] * 4 + [C.c_int]
        fn.restype = C.c_int
    return L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double if a.dtype == np.float64 else C.c_float))


def _ulps(a, b):
    """Distance in units in the last place between same-sign finite arrays."""
    ia = a.view(np.int64 if a.dtype == np.float64 else np.int32).astype(np.int64)
    ib = b.view(np.int64 if b.dtype == np.float64 else np.int32).astype(np.int64)
    return np.abs(ia - ib)


@pytest.mark.parametrize("dtype,fn", [(np.float64, "dm_rcp64"), (np.float32, "dm_rcp32")])
def test_rcp_within_one_ulp_of_ieee_division(dm, dtype, fn):
    rng = np.random.default_rng(7)
    x = np.concatenate([np.logspace(-6, 6, 200001), 10 ** rng.uniform(-6, 6, 200000),
                        [1.0, 2.0, 0.5, 3.0, 1.4, 0.4, 1e-6, 1e6]]).astype(dtype)
    ours, div = np.empty_like(x), np.empty_like(x)
    assert getattr(dm, fn)(_p(x), _p(ours), _p(div), len(x)) == 0
    # CUDA's division is IEEE round-to-nearest, as numpy's
    np.testing.assert_array_equal(div, (dtype(1) / x).astype(dtype))
    assert _ulps(ours, div).max() <= 1


def _exact_log_mean(x, y):
    xl, yl = x.astype(np.longdouble), y.astype(np.longdouble)
    out = np.where(xl == yl, xl, (yl - xl) / (np.log(yl) - np.log(xl)))
    return out


def _ratios(switch_ratio, n=40001):
    """y/x ratios from 1 to 2.5, dense around the branch switch."""
    dense = switch_ratio * (1.0 + np.linspace(-2e-3, 2e-3, n))
    return np.unique(np.concatenate([[1.0], np.linspace(1.0, 2.5, n), dense, 1.0 / dense]))


@pytest.mark.parametrize("dtype,fn,switch_u", [
    (np.float64, "dm_log_mean64", 1e-4),
    (np.float32, "dm_log_mean32", 0.04),
])
def test_log_mean_both_branches(dm, dtype, fn, switch_u):
    """Relative error against the exact mean, bounded pointwise by the
    conditioning of each branch: a few rounding units on the series branch;
    on the logarithm branch the rounding of y/x is amplified by 1/|ln(y/x)|
    (the reference's (y - x)/log(y/x) has the same amplification), so the bound
    there is 3 eps/|ln(y/x)| + 6 eps."""
    eps = float(np.finfo(dtype).eps) / 2
    f = np.sqrt(switch_u)
    ratio = _ratios((1 + f) / (1 - f))
    rng = np.random.default_rng(11)
    x = 10 ** rng.uniform(-2, 2, len(ratio))
    y = x * ratio
    x, y = x.astype(dtype), y.astype(dtype)
    mean, inv = np.empty_like(x), np.empty_like(x)
    assert getattr(dm, fn)(_p(x), _p(y), _p(mean), _p(inv), len(x)) == 0
    ex = _exact_log_mean(x, y)
    rel = np.abs(mean.astype(np.longdouble) - ex) / ex
    rel_inv = np.abs(inv.astype(np.longdouble) * ex - 1)
    xd, yd = x.astype(np.float64), y.astype(np.float64)
    ff = (yd - xd) / (yd + xd)
    u = ff * ff
    # the branch a point takes; within 0.1 % of the switch either may be taken
    series = u < switch_u * (1 - 1e-3)
    other = ~series
    assert series.any() and (u > switch_u * (1 + 1e-3)).any(), "the sweep must cover both branches"
    assert float(rel[series].max()) <= 12 * eps
    assert float(rel_inv[series].max()) <= 12 * eps
    lnr = np.abs(np.log(yd[other] / xd[other]))
    bound = 3 * eps / lnr + 12 * eps
    assert bool((rel[other] <= bound).all())
    assert bool((rel_inv[other] <= bound).all())


def test_reference_series_matches_the_exact_mean():
    """BasicOperations.cpp:6-12's series on its branch (u < 1e-4), on the host."""
    f = np.linspace(-0.01, 0.01, 20001)
    x = np.ones_like(f)
    y = (1 + f) / (1 - f)
    u = ((y - x) / (y + x)) ** 2
    ref = (x + y) * 52.5 / (105 + u * (35 + u * (21 + 15 * u)))
    ex = _exact_log_mean(x, y)
    assert float((np.abs(ref - ex) / ex).max()) <= 12 * float(np.finfo(np.float64).eps) / 2
