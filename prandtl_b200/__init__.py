"""B200-native (sm_100a) DGSEM right-hand side and Runge-Kutta step of Prandtl.

Public surface:
  mesh.periodic_box         periodic affine meshes in the C-ABI descriptor form
  cases                     initial conditions of the benchmark workloads
  operator.DGSEMOperator    mirror of Prandtl::DGSEMOperator backed by the C ABI
  build.build               nvcc build of libprandtl_b200.so (in-tree)
"""
from . import cases, mesh  # noqa: F401

__all__ = ["cases", "mesh", "DGSEMOperator"]


def __getattr__(name):
    if name == "DGSEMOperator":
        from .operator import DGSEMOperator
        return DGSEMOperator
    raise AttributeError(name)
