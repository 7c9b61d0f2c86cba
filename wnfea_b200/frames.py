"""Beam-frame model generator for the co-rotational beam path.

The reference builds frames through its STEP / BeamMesher pipeline (out of scope here);
this generator writes the same ``FEAModel`` fields directly: ``mesh_nodes``,
``mesh_elements`` (2-node beams), ``element_properties`` (material + section per beam,
model.py:37-41, 64-66), fully fixed supports and nodal point loads.
"""

from __future__ import annotations

import numpy as np

from .model import FEAModel, LoadDef, MaterialDef, PropertyAssignment, create_fixed_support, create_rectangular_bar


def generate_frame_grid(
    nx: int = 10,
    ny: int = 10,
    spacing: float = 1.0,
    E: float = 200e9,
    nu: float = 0.3,
    width: float = 0.1,
    height: float = 0.1,
    load_range: float = 5e3,
    seed: int = 0,
) -> FEAModel:
    """nx x ny grid of nodes in the z = 0 plane joined by beams along x and y.

    The four corner nodes are fully clamped; every node carries a seeded z-load drawn
    uniformly from [-load_range, load_range] N.  10 x 10 gives 100 nodes and 180 beams.
    """
    xs, ys = np.meshgrid(np.arange(nx) * spacing, np.arange(ny) * spacing, indexing="ij")
    nodes = np.column_stack([xs.ravel(), ys.ravel(), np.zeros(nx * ny)])

    def nid(i, j):
        return i * ny + j

    elems = [(nid(i, j), nid(i + 1, j)) for i in range(nx - 1) for j in range(ny)]
    elems += [(nid(i, j), nid(i, j + 1)) for i in range(nx) for j in range(ny - 1)]
    model = FEAModel()
    model.mesh_nodes = nodes
    model.mesh_elements = np.asarray(elems, dtype=np.int32)
    model.materials["Steel"] = MaterialDef("Steel", E, nu, 2.5e8)
    sec = create_rectangular_bar("Rect", width, height)
    model.sections[sec.name] = sec
    model.element_properties = {e: PropertyAssignment("Steel", sec.name) for e in range(len(elems))}
    for n in (nid(0, 0), nid(nx - 1, 0), nid(0, ny - 1), nid(nx - 1, ny - 1)):
        model.supports.append(create_fixed_support(n, is_geometry_node=False))
    fz = np.random.default_rng(seed).uniform(-load_range, load_range, size=nx * ny)
    for n in range(nx * ny):
        model.loads.append(LoadDef(node_id=n, is_geometry_node=False, fz=float(fz[n])))
    return model


def generate_space_frame(
    nx: int = 10,
    ny: int = 10,
    nz: int = 10,
    spacing: float = 1.0,
    E: float = 200e9,
    nu: float = 0.3,
    width: float = 0.1,
    height: float = 0.1,
    load_range: float = 5e3,
    seed: int = 0,
) -> FEAModel:
    """nx x ny x nz lattice of nodes joined by beams along x, y and z.

    Every node of the z = 0 plane is fully clamped; every node of the top plane carries seeded
    forces fx, fy, fz drawn uniformly from [-load_range, load_range] N.  70 x 70 x 70 gives
    343,000 nodes (2,058,000 DOFs) and 1,014,300 beams.
    """
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    nodes = np.column_stack([i.ravel(), j.ravel(), k.ravel()]).astype(np.float64) * spacing
    nid = np.arange(nx * ny * nz).reshape(nx, ny, nz)
    elems = np.concatenate([
        np.column_stack([nid[:-1, :, :].ravel(), nid[1:, :, :].ravel()]),
        np.column_stack([nid[:, :-1, :].ravel(), nid[:, 1:, :].ravel()]),
        np.column_stack([nid[:, :, :-1].ravel(), nid[:, :, 1:].ravel()]),
    ]).astype(np.int32)
    model = FEAModel()
    model.mesh_nodes = nodes
    model.mesh_elements = elems
    model.materials["Steel"] = MaterialDef("Steel", E, nu, 2.5e8)
    sec = create_rectangular_bar("Rect", width, height)
    model.sections[sec.name] = sec
    prop = PropertyAssignment("Steel", sec.name)
    model.element_properties = {e: prop for e in range(len(elems))}
    for n in nid[:, :, 0].ravel():
        model.supports.append(create_fixed_support(int(n), is_geometry_node=False))
    top = nid[:, :, nz - 1].ravel()
    f = np.random.default_rng(seed).uniform(-load_range, load_range, size=(len(top), 3))
    for n, (fx, fy, fz) in zip(top, f):
        model.loads.append(LoadDef(node_id=int(n), is_geometry_node=False, fx=float(fx), fy=float(fy), fz=float(fz)))
    return model
