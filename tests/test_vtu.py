"""VTU export: the file layout and fields of the reference's exporter, read back with an XML
parser; solid stresses (GPU) against the oracle's stress field."""

from __future__ import annotations

import xml.etree.ElementTree as ET
from types import SimpleNamespace

import numpy as np
import pytest

from wnfea_b200.frames import generate_frame_grid
from wnfea_b200.vtu import export_vtu


def _arrays(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    out = {a.get("Name"): np.array(a.text.split(), dtype=float) for a in piece.iter("DataArray")}
    return piece, out


def test_beam_frame_export(tmp_path):
    m = generate_frame_grid(nx=4, ny=3)
    n = len(m.mesh_nodes)
    U = np.random.default_rng(0).standard_normal(6 * n) * 1e-3
    m.displacements = U
    m.element_results = {e: SimpleNamespace(max_von_mises=1e6 * (e + 1), axial_stress=-1e5 * e)
                         for e in range(len(m.mesh_elements))}
    path = export_vtu(m, tmp_path / "frame.vtu")
    piece, a = _arrays(path)
    nb = len(m.mesh_elements)
    assert piece.get("NumberOfPoints") == str(n) and piece.get("NumberOfCells") == str(nb)
    np.testing.assert_array_equal(a["connectivity"], np.asarray(m.mesh_elements).ravel())
    np.testing.assert_array_equal(a["offsets"], 2 * np.arange(1, nb + 1))
    assert (a["types"] == 3).all()
    np.testing.assert_allclose(a["Points"], np.asarray(m.mesh_nodes).ravel(), rtol=1e-8)
    np.testing.assert_allclose(a["Displacement"], U.reshape(n, 6)[:, :3].ravel(), rtol=1e-8, atol=1e-20)
    np.testing.assert_allclose(a["Rotation"], U.reshape(n, 6)[:, 3:].ravel(), rtol=1e-8, atol=1e-20)
    vm = 1e6 * (np.arange(nb) + 1)
    np.testing.assert_allclose(a["VonMises"], vm, rtol=1e-8)
    np.testing.assert_allclose(a["StressTensor"].reshape(nb, 6)[:, 0], -1e5 * np.arange(nb), rtol=1e-8, atol=1e-20)
    acc = np.zeros(n)
    cnt = np.zeros(n)
    np.add.at(acc, np.asarray(m.mesh_elements).ravel(), np.repeat(vm, 2))
    np.add.at(cnt, np.asarray(m.mesh_elements).ravel(), 1)
    np.testing.assert_allclose(a["VonMises_Nodal"], np.where(cnt > 0, acc / np.maximum(cnt, 1), 0), rtol=1e-8)
    # without results: geometry only
    m.displacements = None
    _, b = _arrays(export_vtu(m, tmp_path / "geom.vtu"))
    assert "VonMises" not in b and not b["Displacement"].any()


@pytest.mark.gpu
def test_solid_export_matches_oracle_stresses(tmp_path):
    from oracle import solid
    from wnfea_b200.mesh import generate_c3d10_kuhn_block
    from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_system

    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    u, _ = solve_c3d10_system(K, F, method="pcg", rtol=1e-10, preconditioner="amg", precision="fp64")
    m.displacements = u
    path = export_vtu(m, tmp_path / "c1.vtu")
    piece, a = _arrays(path)
    ne = len(m.solid_elements)
    assert piece.get("NumberOfCells") == str(ne)
    assert (a["types"] == 24).all()
    np.testing.assert_array_equal(a["offsets"], 10 * np.arange(1, ne + 1))
    props = solid_element_props(m)
    sig, vm, nvm = solid.stress_field(m.mesh_nodes, m.solid_elements, props, u)
    np.testing.assert_allclose(a["VonMises"], vm, rtol=1e-7, atol=1e-7 * vm.max())
    np.testing.assert_allclose(a["StressTensor"].reshape(ne, 6), sig, rtol=0, atol=1e-7 * np.abs(sig).max())
    np.testing.assert_allclose(a["VonMises_Nodal"], nvm, rtol=0, atol=1e-7 * nvm.max())
    np.testing.assert_allclose(a["DisplacementMagnitude"], np.linalg.norm(u.reshape(-1, 3), axis=1), rtol=1e-8,
                               atol=1e-20)
