"""VTK UnstructuredGrid (.vtu, XML, ASCII) export of a model and its results.

Same file layout and field names as the reference's exporter
(wnfea/results/vtu_exporter.py:30-270): C3D10 cells as VTK_QUADRATIC_TETRA (24) and beams as
VTK_LINE (3); point data Displacement, DisplacementMagnitude, Rotation (6-DOF models) and
VonMises_Nodal; cell data VonMises, StressTensor [sxx, syy, szz, sxy, syz, szx] and CellID.
Solid cell stresses are the Gauss-point means computed on the GPU (the stress kernel of
``compute_c3d10_stress_field``); beam cells take ``max_von_mises`` / ``axial_stress`` from
``model.element_results`` when present.  Arrays are formatted in bulk (numpy), not value by
value, so a million-node model writes in seconds.
"""

from __future__ import annotations

import io
from pathlib import Path

import numpy as np

from .model import FEAModel

VTK_LINE = 3
VTK_QUADRATIC_TETRA = 24


def _fmt(values: np.ndarray, fmt: str) -> str:
    buf = io.StringIO()
    np.savetxt(buf, np.asarray(values).reshape(1, -1), fmt=fmt, delimiter=" ")
    return "          " + buf.getvalue().rstrip("\n")


class VTUExporter:
    """Writes FEAModel geometry and results to a .vtu file (reference: vtu_exporter.py:30)."""

    def __init__(self, precision: int = 8):
        self.precision = int(precision)

    def export(self, model: FEAModel, filepath: str | Path, compute_stresses: bool = True) -> str:
        """Write ``model`` to ``filepath``; returns the absolute path (vtu_exporter.py:38-259)."""
        if model.mesh_nodes is None or len(model.mesh_nodes) == 0:
            raise ValueError("FEAModel contains no mesh nodes. Mesh model before exporting.")
        nodes = np.asarray(model.mesh_nodes, dtype=np.float64)
        n_points = len(nodes)
        beams = np.asarray(model.mesh_elements, dtype=np.int64) if model.mesh_elements is not None and len(
            model.mesh_elements) else np.zeros((0, 2), dtype=np.int64)
        solids = np.asarray(model.solid_elements, dtype=np.int64) if getattr(
            model, "solid_elements", None) is not None and len(model.solid_elements) else np.zeros((0, 10), np.int64)
        n_beams, n_solids = len(beams), len(solids)
        n_cells = n_beams + n_solids
        if n_cells == 0:
            raise ValueError("FEAModel has mesh nodes but no beam or solid elements to export.")
        connectivity = np.concatenate([beams.ravel(), solids.ravel()])
        offsets = np.concatenate([2 * np.arange(1, n_beams + 1), 2 * n_beams + 10 * np.arange(1, n_solids + 1)])
        types = np.concatenate([np.full(n_beams, VTK_LINE), np.full(n_solids, VTK_QUADRATIC_TETRA)])

        # point data: translations / rotations from a 3- or 6-DOF displacement vector
        u_trans = np.zeros((n_points, 3))
        u_rot = np.zeros((n_points, 3))
        has_u = model.displacements is not None
        if has_u:
            U = np.asarray(model.displacements, dtype=np.float64).ravel()
            if len(U) == 6 * n_points:
                u_trans, u_rot = U.reshape(n_points, 6)[:, :3], U.reshape(n_points, 6)[:, 3:]
            elif len(U) == 3 * n_points:
                u_trans = U.reshape(n_points, 3)
            else:  # partial vectors: fill what there is at 6 DOFs per node (vtu_exporter.py:117-123)
                tmp = np.zeros(6 * n_points)
                k = min(len(U), 6 * n_points)
                tmp[:k] = U[:k]
                u_trans, u_rot = tmp.reshape(n_points, 6)[:, :3], tmp.reshape(n_points, 6)[:, 3:]
        u_mag = np.linalg.norm(u_trans, axis=1)

        # cell data: solid stresses on the GPU, beam values from element_results
        stresses = has_u and compute_stresses
        cell_vm = np.zeros(n_cells)
        cell_sig = np.zeros((n_cells, 6))
        nodal_vm = np.zeros(n_points)
        if stresses:
            acc = np.zeros(n_points)
            cnt = np.zeros(n_points, dtype=np.int64)
            if n_beams and model.element_results:
                for e in range(n_beams):
                    er = model.element_results.get(e)
                    if er is not None:
                        cell_vm[e] = getattr(er, "max_von_mises", 0.0)
                        cell_sig[e, 0] = getattr(er, "axial_stress", 0.0)
            if n_beams:
                np.add.at(acc, beams.ravel(), np.repeat(cell_vm[:n_beams], 2))
                np.add.at(cnt, beams.ravel(), 1)
            if n_solids:
                from .solid_solver import compute_c3d10_stress_field

                sig, vm, _ = compute_c3d10_stress_field(model, np.ascontiguousarray(u_trans).ravel())
                cell_sig[n_beams:] = sig
                cell_vm[n_beams:] = vm
                np.add.at(acc, solids.ravel(), np.repeat(vm, 10))
                np.add.at(cnt, solids.ravel(), 1)
            m = cnt > 0
            nodal_vm[m] = acc[m] / cnt[m]

        f = f"%.{self.precision}e"
        lines = ['<?xml version="1.0"?>',
                 '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
                 '  <UnstructuredGrid>',
                 f'    <Piece NumberOfPoints="{n_points}" NumberOfCells="{n_cells}">',
                 '      <PointData>']

        def array(name, dtype, values, ncomp=None, fmt=f):
            comp = f' NumberOfComponents="{ncomp}"' if ncomp is not None else ""
            lines.append(f'        <DataArray type="{dtype}" Name="{name}"{comp} format="ascii">')
            lines.append(_fmt(values, fmt))
            lines.append('        </DataArray>')

        array("Displacement", "Float64", u_trans, 3)
        array("DisplacementMagnitude", "Float64", u_mag, 1)
        if has_u and np.any(u_rot != 0.0):
            array("Rotation", "Float64", u_rot, 3)
        if stresses:
            array("VonMises_Nodal", "Float64", nodal_vm, 1)
        lines += ['      </PointData>', '      <CellData>']
        if stresses:
            array("VonMises", "Float64", cell_vm, 1)
            array("StressTensor", "Float64", cell_sig, 6)
        array("CellID", "Int64", np.arange(n_cells), 1, "%d")
        lines += ['      </CellData>', '      <Points>']
        array("Points", "Float64", nodes, 3)
        lines += ['      </Points>', '      <Cells>']
        array("connectivity", "Int64", connectivity, None, "%d")
        array("offsets", "Int64", offsets, None, "%d")
        array("types", "UInt8", types, None, "%d")
        lines += ['      </Cells>', '    </Piece>', '  </UnstructuredGrid>', '</VTKFile>']
        out = Path(filepath).resolve()
        out.parent.mkdir(parents=True, exist_ok=True)
        out.write_text("\n".join(lines) + "\n", encoding="utf-8")
        return str(out)


def export_vtu(model: FEAModel, filepath: str | Path, compute_stresses: bool = True) -> str:
    """Convenience wrapper (vtu_exporter.py:262-270)."""
    return VTUExporter().export(model, filepath, compute_stresses=compute_stresses)
