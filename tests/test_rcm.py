"""RCM renumbering: the node graph equals the element node-pair graph of the reference's
construction, the order cuts the bandwidth of a scrambled mesh, and a solve on the renumbered
model returns the original solution after permute_solution_to_original."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

from wnfea_b200.mesh import generate_c3d10_ibeam_structured
from wnfea_b200.rcm import (apply_rcm_to_model, compute_matrix_bandwidth, compute_node_adjacency_matrix,
                            compute_rcm_order, permute_solution_to_original)


def _scrambled_ibeam(n_slices=8, seed=0):
    m, _ = generate_c3d10_ibeam_structured(n_slices=n_slices, length=4.0 * n_slices / 315, seed=1)
    n = len(m.mesh_nodes)
    perm = np.random.default_rng(seed).permutation(n)  # new -> old: a mesher's arbitrary numbering
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    m.mesh_nodes = m.mesh_nodes[perm].copy()
    m.solid_elements = inv[m.solid_elements].astype(np.int32)
    for s in m.supports:
        if not s.is_geometry_node:
            s.node_id = int(inv[s.node_id])
    for ld in m.loads:
        if not ld.is_geometry_node:
            ld.node_id = int(inv[ld.node_id])
    return m


def test_adjacency_is_the_element_node_pair_graph():
    m = _scrambled_ibeam(4)
    n = len(m.mesh_nodes)
    beams = np.array([[0, 5], [7, 3]])
    adj = compute_node_adjacency_matrix(n, beams, m.solid_elements)
    e = np.asarray(m.solid_elements)
    r = [np.arange(n), beams[:, 0], beams[:, 1]]
    c = [np.arange(n), beams[:, 1], beams[:, 0]]
    for i in range(10):
        for j in range(10):
            if i != j:
                r.append(e[:, i])
                c.append(e[:, j])
    ref = sp.csr_matrix((np.ones(sum(len(x) for x in r)), (np.concatenate(r), np.concatenate(c))), shape=(n, n))
    ref.data[:] = 1
    assert (adj != ref).nnz == 0


def test_rcm_cuts_bandwidth_and_round_trips():
    m = _scrambled_ibeam(8)
    n = len(m.mesh_nodes)
    adj = compute_node_adjacency_matrix(n, None, m.solid_elements)
    new_to_old, old_to_new = compute_rcm_order(adj)
    assert np.array_equal(np.sort(new_to_old), np.arange(n)) and np.array_equal(old_to_new[new_to_old], np.arange(n))
    before = compute_matrix_bandwidth(adj)
    after = compute_matrix_bandwidth(adj[new_to_old][:, new_to_old])
    assert after < 0.1 * before
    u = np.random.default_rng(1).standard_normal(3 * n)
    u_new = u.reshape(n, 3)[new_to_old].ravel()
    assert np.array_equal(permute_solution_to_original(u_new, new_to_old, 3), u)
    with pytest.raises(ValueError):
        permute_solution_to_original(u_new[:-1], new_to_old, 3)


@pytest.mark.gpu
def test_solve_on_renumbered_model_gives_the_same_solution():
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_system

    m = _scrambled_ibeam(8)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    u0, _ = solve_c3d10_system(K, F, method="pcg", rtol=1e-10, preconditioner="amg", precision="fp64")
    mr, new_to_old, _ = apply_rcm_to_model(m)
    Kr, Fr, _ = assemble_c3d10_sparse_3dof(mr)
    assert np.array_equal(permute_solution_to_original(Fr, new_to_old, 3), F)
    ur, _ = solve_c3d10_system(Kr, Fr, method="pcg", rtol=1e-10, preconditioner="amg", precision="fp64")
    u1 = permute_solution_to_original(ur, new_to_old, 3)
    assert np.linalg.norm(u1 - u0) <= 1e-8 * np.linalg.norm(u0)
