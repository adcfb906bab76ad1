"""Checkpoint/resume files and ParaView output (``prandtl_checkpoint_*``,
``prandtl_paraview_save``): the reference's on-disk formats
(``Simulation.cpp:1084-1116``, ``:350-384``, ``:389-410``), written by the
native library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh

_dp = C.POINTER(C.c_double)


def _check(st):
    if st != _lib.PRANDTL_OK:
        raise _lib.PrandtlError(st, _lib.load().prandtl_io_last_error().decode(errors="replace"))


def save_checkpoint(folder: str, cycle: int, time: float, mesh: Mesh, u: np.ndarray, rank: int = 0):
    """Write ``<folder>/Cycle<cycle>/checkpoint_cycle_<cycle>.<rank>.chk`` and its
    JSON meta file (rank 0)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    if u.size != mesh.num_fields * mesh.ndof:
        raise ValueError("state size does not match the mesh")
    _check(_lib.load().prandtl_checkpoint_save(str(folder).encode(), int(cycle), float(time), int(rank), mesh.dim,
                                               mesh.order, mesh.ndof, u.ctypes.data_as(_dp)))


def load_checkpoint(folder: str, cycle: int, mesh: Mesh, rank: int = 0):
    """(state, time) of a checkpoint written by save_checkpoint or by the reference."""
    u = np.empty(mesh.num_fields * mesh.ndof)
    t = C.c_double()
    _check(_lib.load().prandtl_checkpoint_load(str(folder).encode(), int(cycle), int(rank), mesh.dim, mesh.order,
                                               mesh.ndof, u.ctypes.data_as(_dp), C.byref(t)))
    return u, t.value


def save_paraview(folder: str, name: str, cycle: int, time: float, mesh: Mesh, u: np.ndarray, alpha=None,
                  gamma: float = 1.4, binary: bool = True):
    """ParaView collection ``<folder>/<name>/<name>.pvd`` with this cycle added.

    u is the conserved state; for the axisymmetric form pass the recovered U
    (``DGSEMOperator.recover_state(rU)``), as the reference writes its fields
    from it (Simulation.cpp:1041-1044)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    a = None if alpha is None else np.ascontiguousarray(alpha, dtype=np.float64)
    _check(_lib.load().prandtl_paraview_save(str(folder).encode(), str(name).encode(), int(cycle), float(time),
                                             mesh.dim, mesh.order, mesh.num_elements, coords.ctypes.data_as(_dp),
                                             u.ctypes.data_as(_dp), None if a is None else a.ctypes.data_as(_dp),
                                             float(gamma), int(bool(binary))))
