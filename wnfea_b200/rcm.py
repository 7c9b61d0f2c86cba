"""Reverse Cuthill-McKee node renumbering (reference: wnfea/mesh/rcm.py:20-196).

Same functions and conventions as the reference.  The node graph of the C3D10 elements is the
block pattern of the stiffness matrix, so it comes from the library's multithreaded C++ pattern
builder (``wn_bsr3_pattern_host``) instead of a Python enumeration of the 45 node pairs of
every element; beam edges are added on top.  On the GPU the ordering decides how far apart the
x entries gathered by one warp of the block-row SpMV lie: a bandwidth-reducing order keeps a
warp's gathers in few cache lines and the active slice of x resident in L2.
"""

from __future__ import annotations

import copy
import ctypes as C

import numpy as np
import scipy.sparse as sp
import scipy.sparse.csgraph as csg

from . import _lib
from .model import FEAModel


def compute_node_adjacency_matrix(n_nodes: int, beam_elements: np.ndarray | None = None,
                                  solid_elements: np.ndarray | None = None) -> sp.csr_matrix:
    """Symmetric node adjacency with self-loops (rcm.py:20-70), as an int8 CSR matrix."""
    n_nodes = int(n_nodes)
    parts = []
    if solid_elements is not None and len(solid_elements) > 0:
        conn = np.ascontiguousarray(solid_elements, dtype=np.int32)
        nnzb = C.c_int64()
        rp = np.empty(n_nodes + 1, dtype=np.int32)
        _lib.call("wn_bsr3_pattern_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(nnzb), _lib.ptr(rp), None, None)
        ci = np.empty(nnzb.value, dtype=np.int32)
        _lib.call("wn_bsr3_pattern_host", n_nodes, len(conn), _lib.ptr(conn), C.byref(nnzb), _lib.ptr(rp),
                  _lib.ptr(ci), None)
        parts.append(sp.csr_matrix((np.ones(len(ci), dtype=np.int8), ci, rp), shape=(n_nodes, n_nodes)))
    rows = [np.arange(n_nodes)]
    cols = [np.arange(n_nodes)]
    if beam_elements is not None and len(beam_elements) > 0:
        b = np.asarray(beam_elements, dtype=np.int64)
        rows += [b[:, 0], b[:, 1]]
        cols += [b[:, 1], b[:, 0]]
    r, c = np.concatenate(rows), np.concatenate(cols)
    parts.append(sp.csr_matrix((np.ones(len(r), dtype=np.int8), (r, c)), shape=(n_nodes, n_nodes)))
    adj = parts[0]
    for p in parts[1:]:
        adj = adj + p
    adj = sp.csr_matrix(adj)
    adj.data[:] = 1
    adj.sort_indices()
    return adj


def compute_rcm_order(adj: sp.csr_matrix) -> tuple[np.ndarray, np.ndarray]:
    """(new_to_old, old_to_new) of the reverse Cuthill-McKee order (rcm.py:73-92)."""
    new_to_old = np.asarray(csg.reverse_cuthill_mckee(sp.csr_matrix(adj), symmetric_mode=True), dtype=np.int32)
    old_to_new = np.empty(len(new_to_old), dtype=np.int32)
    old_to_new[new_to_old] = np.arange(len(new_to_old), dtype=np.int32)
    return new_to_old, old_to_new


def compute_matrix_bandwidth(A: sp.spmatrix) -> int:
    """Half-bandwidth max |i - j| over the nonzeros (rcm.py:95-102)."""
    r, c = A.nonzero()
    return int(np.max(np.abs(r - c))) if len(r) else 0


def apply_rcm_to_model(model: FEAModel) -> tuple[FEAModel, np.ndarray, np.ndarray]:
    """A renumbered shallow copy of ``model`` with (new_to_old, old_to_new) (rcm.py:105-163):
    coordinates, beam and solid connectivity, and the mesh-node supports and loads follow the
    new numbering; geometry-node references are left as they are."""
    if model.mesh_nodes is None or len(model.mesh_nodes) == 0:
        raise ValueError("Cannot apply RCM to an unmeshed model.")
    n = len(model.mesh_nodes)
    adj = compute_node_adjacency_matrix(n, model.mesh_elements, getattr(model, "solid_elements", None))
    new_to_old, old_to_new = compute_rcm_order(adj)
    out = copy.copy(model)
    out.mesh_nodes = np.asarray(model.mesh_nodes)[new_to_old].copy()
    if model.mesh_elements is not None and len(model.mesh_elements) > 0:
        out.mesh_elements = old_to_new[np.asarray(model.mesh_elements)].copy()
    if getattr(model, "solid_elements", None) is not None and len(model.solid_elements) > 0:
        out.solid_elements = old_to_new[np.asarray(model.solid_elements)].copy()
    out.supports = []
    for s in model.supports:
        c = copy.deepcopy(s)
        if not c.is_geometry_node:
            c.node_id = int(old_to_new[c.node_id])
        out.supports.append(c)
    out.loads = []
    for ld in model.loads:
        c = copy.deepcopy(ld)
        if not c.is_geometry_node:
            c.node_id = int(old_to_new[c.node_id])
        out.loads.append(c)
    if getattr(model, "displacements", None) is not None:
        out.displacements = None  # results of the old numbering do not carry over
    for attr in ("_wn_batch", "_wn_system"):
        if attr in out.__dict__:
            del out.__dict__[attr]
    return out, new_to_old, old_to_new


def permute_solution_to_original(u_permuted: np.ndarray, new_to_old: np.ndarray, dofs_per_node: int = 6) -> np.ndarray:
    """A solution of the renumbered model in the original node numbering (rcm.py:166-196)."""
    u = np.asarray(u_permuted).ravel()
    n = len(new_to_old)
    if len(u) != n * dofs_per_node:
        raise ValueError(f"Length of u_permuted ({len(u)}) does not match {n} nodes * {dofs_per_node} DOFs.")
    idx = (np.asarray(new_to_old)[:, None] * dofs_per_node + np.arange(dofs_per_node)).ravel()
    out = np.empty_like(u)
    out[idx] = u
    return out
