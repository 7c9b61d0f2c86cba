"""Structured C3D10 mesh generators for the solve path's workloads.

``generate_c3d10_structured_block`` is the reference's structured generator
(wnfea/mesh/solid_generator.py:21-213; 5 tets per hex) with the same arguments and the same
mesh node for node, vectorised.  The reference's I-beam generator (solid_generator.py:284-412)
needs Gmsh; the workloads here want a 6-tet (Kuhn) split and a structured I-beam with seeded
jitter, so those generators are new.  All keep the reference's conventions:

* C3D10 node order: 4 corners, then mid-edges 1-2, 2-3, 3-1, 1-4, 2-4, 3-4
  (c3d10.py:52-58 and the edge list at solid_generator.py:131-138);
* a tet with negative signed volume has its 2nd and 3rd corners swapped
  (solid_generator.py:113-115);
* clamp = ``create_fixed_support`` on every node of the root face; loads are equal nodal
  point loads on the tip face (solid_generator.py:176-195).

Kuhn's 6-tet split uses the hex diagonal v000-v111 and the face diagonals that run with
it, so every vertex and every mid-edge node of the mesh lies on the grid of half-cell
points.  Nodes are numbered lexicographically on that half grid, x slowest, which gives
the assembled matrix a narrow band without any reordering.
"""

from __future__ import annotations

from itertools import permutations

import numpy as np

from .model import FEAModel, LoadDef, MaterialDef, create_fixed_support

# corner offsets of a unit hex, as half-grid steps (0 or 2)
_EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))


def _kuhn_tets():
    """The 6 Kuhn tets of a unit cube as (4, 3) corner offsets in {0, 1}."""
    tets = []
    for perm in permutations(range(3)):
        v = np.zeros(3, dtype=np.int64)
        verts = [v.copy()]
        for ax in perm:
            v[ax] += 1
            verts.append(v.copy())
        tets.append(np.array(verts))
    return np.array(tets)  # (6, 4, 3)


def _signed_volume6(p):
    d1 = p[:, 1] - p[:, 0]
    d2 = p[:, 2] - p[:, 0]
    d3 = p[:, 3] - p[:, 0]
    return np.einsum("ij,ij->i", d1, np.cross(d2, d3))


def _build_tets(cells: np.ndarray, xs, ys, zs):
    """C3D10 connectivity (in half-grid index triples) for the hex cells ``cells`` (n, 3).

    Returns half-grid integer coordinates of the 10 nodes of every tet, shape (6n, 10, 3).
    """
    kuhn = _kuhn_tets()  # (6, 4, 3)
    corners = 2 * (cells[:, None, None, :] + kuhn[None, :, :, :])  # (n, 6, 4, 3)
    corners = corners.reshape(-1, 4, 3)
    # orientation on the undistorted grid: swap corners 1 and 2 when the volume is negative
    pts = np.stack([xs[corners[..., 0] // 2], ys[corners[..., 1] // 2], zs[corners[..., 2] // 2]], axis=-1)
    neg = _signed_volume6(pts) < 0.0
    c = corners.copy()
    c[neg, 1], c[neg, 2] = corners[neg, 2], corners[neg, 1]
    mids = np.stack([(c[:, a] + c[:, b]) // 2 for a, b in _EDGES], axis=1)
    return np.concatenate([c, mids], axis=1)  # (6n, 10, 3)


def _half_coords(g):
    """Half-grid coordinates from cell breaks ``g`` (length m+1) -> length 2m+1."""
    g = np.asarray(g, dtype=np.float64)
    h = np.empty(2 * len(g) - 1)
    h[0::2] = g
    h[1::2] = 0.5 * (g[:-1] + g[1:])
    return h


def _number_nodes(tets_hg: np.ndarray, shape):
    """Compact lexicographic (x slowest) numbering of the half-grid points in use."""
    nx, ny, nz = shape
    lin = (tets_hg[..., 0] * ny + tets_hg[..., 1]) * nz + tets_hg[..., 2]
    used = np.unique(lin)
    conn = np.searchsorted(used, lin).astype(np.int32)
    I = used // (ny * nz)
    J = (used // nz) % ny
    K = used % nz
    return conn, np.stack([I, J, K], axis=1)


def _finish_model(coords, conn, E, nu, root_mask, tip_mask, tip_force):
    model = FEAModel()
    model.mesh_nodes = coords
    model.solid_elements = conn
    model.materials["Steel"] = MaterialDef(name="Steel", youngs_modulus=E, poissons_ratio=nu, yield_strength=2.5e8)
    model.solid_materials = {}
    for nid in np.nonzero(root_mask)[0]:
        model.supports.append(create_fixed_support(int(nid), is_geometry_node=False))
    tip = np.nonzero(tip_mask)[0]
    if tip_force is not None and len(tip):
        f = np.asarray(tip_force, dtype=np.float64) / len(tip)
        for nid in tip:
            model.loads.append(LoadDef(node_id=int(nid), is_geometry_node=False, fx=f[0], fy=f[1], fz=f[2]))
    return model


def check_positive_jacobians(coords: np.ndarray, conn: np.ndarray) -> float:
    """Smallest corner-tet signed volume (x6); raises if any element is inverted.

    Mirrors the ``det_J <= 0`` rejection of c3d10.py:129-134 at the corner-tet level; the
    mid-edge nodes generated here are exact midpoints, so the element map is affine and
    its Jacobian is constant and equal to this volume.
    """
    v = _signed_volume6(coords[conn[:, :4]])
    vmin = float(v.min()) if len(v) else 1.0
    if vmin <= 0.0:
        raise ValueError(f"inverted C3D10 element (min 6*volume {vmin:.3e})")
    return vmin


# The reference's 5-tet splitting of a hex (solid_generator.py:66-80), corners numbered
# 0 (i,j,k), 1 (i+1,j,k), 2 (i+1,j+1,k), 3 (i,j+1,k), 4-7 the same at k+1; the two mirror
# splittings alternate with the parity of i + j + k so that neighbouring hexes share their face
# diagonals.  The table and the mid-edge order above must be the reference's for the same mesh.
_HEX5 = np.array([[(0, 1, 3, 4), (1, 2, 3, 6), (1, 4, 5, 6), (3, 4, 6, 7), (1, 3, 4, 6)],
                  [(0, 1, 2, 5), (0, 2, 3, 7), (0, 4, 5, 7), (2, 5, 6, 7), (0, 2, 5, 7)]], dtype=np.int64)


def generate_c3d10_structured_block(length: float = 10.0, width: float = 1.0, height: float = 1.0, nx: int = 40,
                                    ny: int = 4, nz: int = 4, E: float = 2.1e11, nu: float = 0.3,
                                    tip_load_total: float = 10000.0):
    """The reference's structured C3D10 cantilever (wnfea/mesh/solid_generator.py:21-213), the
    same mesh node for node: an (nx, ny, nz) hex grid of the box [0, length] x [0, width] x
    [0, height], each hex cut into 5 tets (parity-alternating splitting), corners numbered
    i (ny+1)(nz+1) + j (nz+1) + k, a tet of negative volume with its 2nd and 3rd corners swapped,
    mid-edge nodes numbered after the corners in order of first use (element by element, edges
    1-2, 2-3, 3-1, 1-4, 2-4, 3-4); the face x = 0 clamped, ``tip_load_total`` shared equally as
    +y forces by the nodes of the face x = length.  Vectorised (no per-element Python loop).
    Returns (model, meta) with the reference's meta keys."""
    import time

    t0 = time.perf_counter()
    xs, ys, zs = np.linspace(0.0, length, nx + 1), np.linspace(0.0, width, ny + 1), np.linspace(0.0, height, nz + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    corners = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    n_corner = len(corners)
    sj, si = nz + 1, (ny + 1) * (nz + 1)
    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = (I * si + J * sj + K).ravel()
    hexc = base[:, None] + np.array([0, si, si + sj, sj, 1, si + 1, si + sj + 1, sj + 1], dtype=np.int64)[None, :]
    parity = ((I + J + K) % 2).ravel()
    tets = np.take_along_axis(hexc[:, None, :], _HEX5[parity].reshape(len(base), 5 * 4)[:, None, :], axis=2)
    tets = tets.reshape(-1, 4)
    neg = _signed_volume6(corners[tets]) < 0.0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    n_el = len(tets)
    # mid-edge nodes in order of first use
    a = np.stack([tets[:, e0] for e0, _ in _EDGES], axis=1).ravel()
    b = np.stack([tets[:, e1] for _, e1 in _EDGES], axis=1).ravel()
    key = np.minimum(a, b) * n_corner + np.maximum(a, b)
    uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty(len(uniq), dtype=np.int64)
    rank[order] = np.arange(len(uniq))
    conn = np.empty((n_el, 10), dtype=np.int32)
    conn[:, :4] = tets
    conn[:, 4:] = (n_corner + rank[inv]).reshape(n_el, 6)
    fa, fb = a[first[order]], b[first[order]]
    coords = np.vstack([corners, 0.5 * (corners[fa] + corners[fb])])
    tol = 1e-6 * length
    root = coords[:, 0] <= tol
    tip = coords[:, 0] >= length - tol
    model = _finish_model(coords, conn, E, nu, root, tip, (0.0, tip_load_total, 0.0))
    model.solid_materials = {i: "Steel" for i in range(n_el)}
    meta = {"length": length, "width": width, "height": height, "grid": (nx, ny, nz), "n_nodes": len(coords),
            "n_elements": n_el, "n_dofs": 3 * len(coords), "root_nodes_fixed": int(root.sum()),
            "tip_nodes_loaded": int(tip.sum()), "build_time_sec": time.perf_counter() - t0}
    return model, meta


def generate_c3d10_kuhn_block(
    length: float = 1.0,
    width: float = 0.1,
    height: float = 0.1,
    nx: int = 20,
    ny: int = 2,
    nz: int = 2,
    E: float = 2.1e11,
    nu: float = 0.3,
    tip_force=(0.0, 0.0, -1000.0),
    clamp: str = "x0",
) -> tuple[FEAModel, dict]:
    """Box [0,length]x[0,width]x[0,height], nx*ny*nz hexes x 6 Kuhn tets = 6*nx*ny*nz C3D10.

    ``clamp="x0"``: every node at x = 0 fixed, ``tip_force`` (total, N) shared equally over
    the nodes at x = length (the cantilever).  ``clamp="z0"``: the z = 0 face fixed and the
    total ``tip_force`` shared over the z = height face (the pressure-loaded block).
    """
    cells = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    xs = np.linspace(0.0, length, nx + 1)
    ys = np.linspace(0.0, width, ny + 1)
    zs = np.linspace(0.0, height, nz + 1)
    tets = _build_tets(cells, xs, ys, zs)
    conn, hg = _number_nodes(tets, (2 * nx + 1, 2 * ny + 1, 2 * nz + 1))
    hx, hy, hz = _half_coords(xs), _half_coords(ys), _half_coords(zs)
    coords = np.stack([hx[hg[:, 0]], hy[hg[:, 1]], hz[hg[:, 2]]], axis=1)
    check_positive_jacobians(coords, conn)
    if clamp == "x0":
        root, tip = hg[:, 0] == 0, hg[:, 0] == 2 * nx
    elif clamp == "z0":
        root, tip = hg[:, 2] == 0, hg[:, 2] == 2 * nz
    else:
        raise ValueError(f"unknown clamp {clamp!r}")
    model = _finish_model(coords, conn, E, nu, root, tip, tip_force)
    meta = {
        "n_nodes": len(coords),
        "n_elements": len(conn),
        "n_dofs": 3 * len(coords),
        "grid": (nx, ny, nz),
        "root_nodes_fixed": int(root.sum()),
        "tip_nodes_loaded": int(tip.sum()),
    }
    return model, meta


def _breaks(segments):
    """Concatenate (length, n_cells) segments into one strictly increasing break list."""
    out = [0.0]
    for seg_len, n in segments:
        start = out[-1]
        out.extend(start + seg_len * (np.arange(1, n + 1) / n))
    return np.asarray(out)


def generate_c3d10_ibeam_structured(
    length: float = 4.0,
    flange_width: float = 0.2,
    flange_thickness: float = 0.02,
    web_thickness: float = 0.015,
    height: float = 0.3,
    n_slices: int = 315,
    flange_half_cells: int = 7,
    web_y_cells: int = 2,
    flange_z_cells: int = 2,
    web_z_cells: int = 21,
    jitter: float = 0.05,
    seed: int = 0,
    E: float = 2.1e11,
    nu: float = 0.3,
    tip_force=(0.0, 0.0, -50_000.0),
) -> tuple[FEAModel, dict]:
    """Structured I-beam along x, 6 Kuhn tets per hex, seeded corner-node jitter.

    Cross-section in (y, z): flanges ``flange_width`` x ``flange_thickness`` at the bottom and
    top, web ``web_thickness`` wide between them (total ``height``).  y cells: 7 per flange
    half, 2 through the web; z cells: 2 per flange, 21 through the web; that is 106 cells per
    slice, and 315 slices give 200,340 C3D10 elements.  Corner nodes strictly inside the
    solid move by a seeded uniform offset of up to ``jitter`` x the local cell size along each
    axis; boundary nodes move only along x and never off the root or tip plane, so every face
    stays planar.  Mid-edge nodes are the midpoints of their (moved) corners.  Root x = 0
    clamped; ``tip_force`` (total) shared equally over the x = length nodes.
    """
    half_out = 0.5 * (flange_width - web_thickness)
    ys = _breaks([(half_out, flange_half_cells), (web_thickness, web_y_cells), (half_out, flange_half_cells)])
    web_h = height - 2.0 * flange_thickness
    zs = _breaks([(flange_thickness, flange_z_cells), (web_h, web_z_cells), (flange_thickness, flange_z_cells)])
    xs = np.linspace(0.0, length, n_slices + 1)
    ys = ys - 0.5 * flange_width  # centre the section on y = 0
    ny, nz = len(ys) - 1, len(zs) - 1
    jy0, jy1 = flange_half_cells, flange_half_cells + web_y_cells  # web y-cell range
    present = np.zeros((ny, nz), dtype=bool)
    present[:, :flange_z_cells] = True
    present[:, nz - flange_z_cells:] = True
    present[jy0:jy1, :] = True
    jk = np.argwhere(present)
    cells = np.concatenate([np.column_stack([np.full(len(jk), i), jk]) for i in range(n_slices)])
    tets = _build_tets(cells, xs, ys, zs)
    conn, hg = _number_nodes(tets, (2 * n_slices + 1, 2 * ny + 1, 2 * nz + 1))
    hx, hy, hz = _half_coords(xs), _half_coords(ys), _half_coords(zs)
    coords = np.stack([hx[hg[:, 0]], hy[hg[:, 1]], hz[hg[:, 2]]], axis=1)

    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        corner = np.all(hg % 2 == 0, axis=1)
        ci = hg // 2  # cell-break indices of corner nodes
        # interior test: all 4 surrounding section cells present and the node not on x=0/L
        jj, kk = ci[:, 1], ci[:, 2]
        inside = np.ones(len(hg), dtype=bool)
        for dj in (-1, 0):
            for dk in (-1, 0):
                j, k = jj + dj, kk + dk
                ok = (j >= 0) & (j < ny) & (k >= 0) & (k < nz)
                pres = np.zeros(len(hg), dtype=bool)
                pres[ok] = present[j[ok], k[ok]]
                inside &= pres
        on_x_plane = (ci[:, 0] == 0) | (ci[:, 0] == n_slices)
        dx = xs[1] - xs[0]
        dyc = np.diff(ys)
        dzc = np.diff(zs)
        loc_dy = np.minimum(dyc[np.clip(jj - 1, 0, ny - 1)], dyc[np.clip(jj, 0, ny - 1)])
        loc_dz = np.minimum(dzc[np.clip(kk - 1, 0, nz - 1)], dzc[np.clip(kk, 0, nz - 1)])
        r = rng.uniform(-1.0, 1.0, size=(len(hg), 3)) * jitter
        move_x = corner & ~on_x_plane
        move_yz = corner & inside & ~on_x_plane
        coords[move_x, 0] += r[move_x, 0] * dx
        coords[move_yz, 1] += r[move_yz, 1] * loc_dy[move_yz]
        coords[move_yz, 2] += r[move_yz, 2] * loc_dz[move_yz]
        # mid-edge nodes: midpoints of their element edge's (moved) corners
        for e_idx, (a, b) in enumerate(_EDGES):
            m = conn[:, 4 + e_idx]
            coords[m] = 0.5 * (coords[conn[:, a]] + coords[conn[:, b]])
    check_positive_jacobians(coords, conn)
    root, tip = hg[:, 0] == 0, hg[:, 0] == 2 * n_slices
    model = _finish_model(coords, conn, E, nu, root, tip, tip_force)
    meta = {
        "n_nodes": len(coords),
        "n_elements": len(conn),
        "n_dofs": 3 * len(coords),
        "cells_per_slice": int(present.sum()),
        "n_slices": n_slices,
        "root_nodes_fixed": int(root.sum()),
        "tip_nodes_loaded": int(tip.sum()),
    }
    return model, meta


def tip_load_cases(coords: np.ndarray, n_cases: int = 32, seed: int = 0, f_min: float = 1e4, f_max: float = 1e5,
                   axis: int = 0) -> np.ndarray:
    """Seeded batch of tip load cases (3 n_nodes, n_cases): case j is a total force of magnitude
    U[f_min, f_max] along a direction uniform on the unit sphere (a normalised Gaussian),
    shared equally over the nodes of the far end (coords[:, axis] == max)."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n_cases, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    mag = rng.uniform(f_min, f_max, size=n_cases)
    x = coords[:, axis]
    tip = np.flatnonzero(x >= x.max() - 1e-9 * max(1.0, abs(x.max())))
    F = np.zeros((3 * len(coords), n_cases))
    for c in range(3):
        F[3 * tip + c, :] = (d[:, c] * mag / len(tip))[None, :]
    return F


# face corner triples of a C3D10 (local indices) and their mid-edge nodes
_FACES = (((0, 1, 2), (4, 5, 6)), ((0, 1, 3), (4, 8, 7)), ((1, 2, 3), (5, 9, 8)), ((0, 2, 3), (6, 9, 7)))


def face_pressure_loads(coords: np.ndarray, conn: np.ndarray, axis: int, value: float, pressure: float,
                        tol: float = 1e-9) -> np.ndarray:
    """Consistent nodal forces (n, 3) of a uniform pressure on the element faces lying in the
    plane coords[:, axis] == value, pushing towards -axis for pressure > 0.

    A flat quadratic (6-node) triangle of area A under uniform traction t carries 0 at its
    corners and t A / 3 at each mid-edge node (the integrals of the quadratic triangle's
    shape functions).
    """
    F = np.zeros((len(coords), 3))
    on = np.abs(coords[:, axis] - value) <= tol * max(1.0, abs(value))
    for corners, mids in _FACES:
        c = conn[:, corners]
        sel = on[c].all(axis=1)
        if not sel.any():
            continue
        p = coords[c[sel]]
        area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)
        m = conn[sel][:, mids]
        np.add.at(F[:, axis], m.ravel(), np.repeat(-pressure * area / 3.0, 3))
    return F


def generate_c3d10_pressure_block(
    length: float = 2.0,
    width: float = 1.0,
    height: float = 0.5,
    nx: int = 60,
    ny: int = 30,
    nz: int = 15,
    e_min: float = 1e9,
    e_max: float = 210e9,
    nu: float = 0.3,
    pressure: float = 10e3,
    seed: int = 0,
) -> tuple[FEAModel, dict]:
    """Kuhn block (6 tets per hex) with per-element E log-uniform in [e_min, e_max] (seeded),
    the z = 0 face clamped and a uniform pressure on the z = height face, applied as
    consistent quadratic-face nodal loads.  60 x 30 x 15 hexes give 162,000 elements."""
    model, meta = generate_c3d10_kuhn_block(length, width, height, nx, ny, nz, E=e_max, nu=nu, tip_force=None,
                                            clamp="z0")
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(np.log(e_min), np.log(e_max), size=len(model.solid_elements)))
    model.solid_props = np.column_stack([E, np.full_like(E, nu)])
    F = face_pressure_loads(model.mesh_nodes, model.solid_elements, 2, height, pressure)
    model.loads = [LoadDef(node_id=int(i), is_geometry_node=False, fx=F[i, 0], fy=F[i, 1], fz=F[i, 2])
                   for i in np.nonzero(np.abs(F).sum(axis=1))[0]]
    meta["total_load"] = float(F[:, 2].sum())
    return model, meta
