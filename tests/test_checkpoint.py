"""Checkpoint/resume and ParaView output files (prandtl_checkpoint_*, prandtl_paraview_save).

File layout and formats follow the reference's Simulation.cpp (checkpoints
:1084-1116 / :350-384, ParaView :389-410).  Round trips are exact; a resumed
oracle trajectory equals the uninterrupted one bit for bit; the VTU cells
hold the state interpolated to their equispaced Lagrange points.
"""
import base64
import json
import os
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from prandtl_b200 import _lib, cases
from prandtl_b200.checkpoint import load_checkpoint, save_checkpoint, save_paraview
from prandtl_b200.mesh import periodic_box


def test_checkpoint_files_and_exact_round_trip(tmp_path):
    mesh = periodic_box(2, 3, 3, 0.0, 1.0)
    u = cases.perturbed(mesh, cases.free_stream(mesh), amp=0.2, seed=3)
    save_checkpoint(tmp_path, 40, 0.123456789012345678, mesh, u)
    save_checkpoint(tmp_path, 40, 0.123456789012345678, mesh, u, rank=3)
    d = tmp_path / "Cycle40"
    assert sorted(os.listdir(d)) == ["checkpoint_cycle_40.00000000.chk", "checkpoint_cycle_40.00000003.chk",
                                     "checkpoint_cycle_40.json"]
    meta = json.loads((d / "checkpoint_cycle_40.json").read_text())
    assert meta == {"time": 0.12345678901234568, "cycle": 40}
    head = (d / "checkpoint_cycle_40.00000000.chk").read_text().split("\n")[:5]
    assert head == ["FiniteElementSpace", "FiniteElementCollection: L2_T1_2D_P3", "VDim: 4", "Ordering: 0", ""]
    v, t = load_checkpoint(tmp_path, 40, mesh)
    assert np.array_equal(v, u) and t == 0.12345678901234568


def test_loads_reference_precision_and_ordering(tmp_path):
    """The reference's own files keep 6 significant digits (default stream
    precision) and may be byVDIM; both load."""
    mesh = periodic_box(2, 2, 2, 0.0, 1.0)
    u = cases.perturbed(mesh, cases.free_stream(mesh), amp=0.2, seed=4)
    nf, n = mesh.num_fields, mesh.ndof
    d = tmp_path / "Cycle7"
    d.mkdir()
    (d / "checkpoint_cycle_7.json").write_text('{\n "time": 0.250000,\n "cycle": 7\n}\n')
    vals = u.reshape(nf, n).T.reshape(-1)   # byVDIM
    (d / "checkpoint_cycle_7.00000000.chk").write_text(
        "FiniteElementSpace\nFiniteElementCollection: L2_T1_2D_P2\nVDim: 4\nOrdering: 1\n\n" +
        "\n".join(f"{x:g}" for x in vals) + "\n")
    v, t = load_checkpoint(tmp_path, 7, mesh)
    assert t == 0.25
    np.testing.assert_allclose(v, u, rtol=1e-5)


def test_checkpoint_errors(tmp_path):
    mesh = periodic_box(2, 2, 2, 0.0, 1.0)
    u = cases.free_stream(mesh)
    save_checkpoint(tmp_path, 5, 1.0, mesh, u)
    with pytest.raises(_lib.PrandtlError):
        load_checkpoint(tmp_path, 6, mesh)                      # no such cycle
    with pytest.raises(_lib.PrandtlError):
        load_checkpoint(tmp_path, 5, periodic_box(2, 2, 3, 0.0, 1.0))   # another order
    (tmp_path / "Cycle5" / "checkpoint_cycle_5.json").write_text('{"time": 1.0, "cycle": 4}')
    with pytest.raises(_lib.PrandtlError):
        load_checkpoint(tmp_path, 5, mesh)                      # meta cycle mismatch
    save_checkpoint(tmp_path, 0, 0.0, mesh, u)
    with pytest.raises(_lib.PrandtlError):
        load_checkpoint(tmp_path, 0, mesh)                      # the reference requires cycle > 0


def test_resume_equals_uninterrupted_run(oracle_mod, tmp_path):
    mesh = periodic_box(2, 4, 3, 0.0, 10.0)
    u0 = cases.isentropic_vortex(mesh)
    orc = oracle_mod.Oracle(mesh, quirks=1)
    dt = 0.4 * mesh.hmin / (orc.rhs(u0)["lambda_max"] * 16)
    full = orc.step(u0, dt, scheme=0, nsteps=6)
    half = orc.step(u0, dt, scheme=0, nsteps=3)
    save_checkpoint(tmp_path, 3, 3 * dt, mesh, half)
    u, t = load_checkpoint(tmp_path, 3, mesh)
    assert t == 3 * dt
    assert np.array_equal(orc.step(u, dt, scheme=0, nsteps=3), full)


def _read_vtu(path):
    root = ET.parse(path).getroot()
    out = {}
    for da in root.iter("DataArray"):
        raw = base64.b64decode(da.text.strip())
        nb = struct.unpack("<I", raw[:4])[0]
        fmt = {"Float64": "d", "Int64": "q", "UInt8": "B"}[da.get("type")]
        out[da.get("Name")] = np.frombuffer(raw[4:4 + nb], dtype=np.dtype(fmt).newbyteorder("<"))
    return out


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 3), (3, 2), (3, 4)])
def test_paraview_cells(tmp_path, dim, order):
    mesh = periodic_box(dim, 2, order, 0.0, 1.0, affine=np.eye(dim) + 0.1 * np.eye(dim, k=1))
    x = mesh.coords
    # a polynomial of degree <= order per direction: interpolation is exact
    rho = 1.0 + 0.1 * x[0] ** order + 0.05 * x[1]
    vel = [0.2 + 0.1 * x[1], -0.1 * x[0], 0.05 + 0.0 * x[0]][:dim]
    p = 1.0 + 0.2 * x[0] * x[1] if order >= 2 else 1.0 + 0.2 * x[0]
    E = p / 0.4 + 0.5 * rho * sum(v * v for v in vel)
    u = np.concatenate([rho, *[rho * v for v in vel], E])
    alpha = np.linspace(0.0, 0.5, mesh.num_elements)
    save_paraview(tmp_path, "out", 0, 0.0, mesh, u, alpha)
    save_paraview(tmp_path, "out", 12, 0.5, mesh, u, alpha)
    save_paraview(tmp_path, "out", 12, 0.5, mesh, u, alpha)   # rewritten, not duplicated
    pvd = (tmp_path / "out" / "out.pvd").read_text()
    assert pvd.count("<DataSet") == 2 and "Cycle000012/data.pvtu" in pvd
    assert (tmp_path / "out" / "Cycle000012" / "data.pvtu").exists()
    d = _read_vtu(tmp_path / "out" / "Cycle000012" / "proc000000.vtu")
    ND = (order + 1) ** dim
    assert d["types"].tolist() == [70 if dim == 2 else 72] * mesh.num_elements
    assert d["offsets"][-1] == mesh.num_elements * ND
    P = d["Points"].reshape(-1, 3)[:, :dim]
    # every point a lattice point of its element, all distinct within an element
    for e in range(mesh.num_elements):
        pe = P[e * ND:(e + 1) * ND]
        assert len({tuple(np.round(q, 10)) for q in pe}) == ND
    # fields are the polynomial evaluated at the points
    xx = P.T
    rho_p = 1.0 + 0.1 * xx[0] ** order + 0.05 * xx[1]
    np.testing.assert_allclose(d["Density"], rho_p, rtol=0, atol=1e-12)
    np.testing.assert_allclose(d["Horizontal V"], 0.2 + 0.1 * xx[1], rtol=0, atol=1e-9)
    assert ("Normal V" in d) == (dim == 3)
    np.testing.assert_allclose(d["Blending Coeff"], np.repeat(alpha, ND))
    # corners of each cell come first, in VTK's corner order
    for e in range(mesh.num_elements):
        c = P[e * ND:e * ND + 4]
        lo = x[:, e * ND:(e + 1) * ND]
        n0 = lo[:, 0]
        nN = lo[:, order]   # node (N, 0[, 0])
        np.testing.assert_allclose(c[0], n0, atol=1e-12)
        np.testing.assert_allclose(c[1], nN, atol=1e-12)
