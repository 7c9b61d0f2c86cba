"""The reference-named structured C3D10 generator against the reference's own output.

``generate_c3d10_structured_block`` (wnfea/mesh/solid_generator.py:21-213) is how the
reference's solid test builds its mesh (tests/test_solid_bench.py:18-26); the drop-in must give
the same mesh node for node, since node numbers appear in the caller's supports, loads and
results.  Pinned against tests/golden/structured_block.npz (made by running the reference's
generator, tests/golden/make_golden.py): coordinates, connectivity, clamped and loaded nodes
with their loads and the meta counts, bit for bit; and the oracle's assembly on our mesh gives
the reference's F and fixed DOFs.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import solid
from wnfea_b200.mesh import check_positive_jacobians, generate_c3d10_structured_block
from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector


@pytest.fixture(scope="module")
def block():
    g = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "structured_block.npz")
    m, meta = generate_c3d10_structured_block(length=5.0, width=1.0, height=1.0, nx=10, ny=3, nz=3,
                                              tip_load_total=1000.0)
    return g, m, meta


def test_structured_block_is_the_reference_mesh(block):
    g, m, meta = block
    assert np.array_equal(m.mesh_nodes, g["nodes"])
    assert np.array_equal(m.solid_elements, g["conn"])
    assert np.array_equal([s.node_id for s in m.supports], g["fixed_nodes"])
    assert np.array_equal([ld.node_id for ld in m.loads], g["load_nodes"])
    assert np.array_equal([[ld.fx, ld.fy, ld.fz] for ld in m.loads], g["load_f"])
    assert [meta[k] for k in ("n_nodes", "n_elements", "n_dofs", "root_nodes_fixed", "tip_nodes_loaded")] == \
        list(g["counts"])
    assert len(m.solid_materials) == meta["n_elements"]
    check_positive_jacobians(m.mesh_nodes, m.solid_elements)


def test_structured_block_loads_and_supports(block):
    g, m, _ = block
    assert np.array_equal(solid_load_vector(m), g["F"])
    assert np.array_equal(np.sort(np.asarray(solid_fixed_dofs(m), dtype=np.int64)), np.sort(g["fixed"]))


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 1, 3), (5, 2, 2)])
def test_structured_block_small_grids(n):
    """Every grid: 5 tets per hex, conforming (each interior face shared by exactly two tets),
    positive Jacobians, mid-edge nodes at the edge midpoints."""
    m, meta = generate_c3d10_structured_block(length=2.0, width=1.0, height=0.5, nx=n[0], ny=n[1], nz=n[2])
    conn, X = m.solid_elements, m.mesh_nodes
    assert meta["n_elements"] == 5 * n[0] * n[1] * n[2] == len(conn)
    check_positive_jacobians(X, conn)
    for k, (a, b) in enumerate(((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))):
        assert np.array_equal(X[conn[:, 4 + k]], 0.5 * (X[conn[:, a]] + X[conn[:, b]]))
    faces = np.sort(np.concatenate([conn[:, [0, 1, 2]], conn[:, [0, 1, 3]], conn[:, [1, 2, 3]], conn[:, [0, 2, 3]]]),
                    axis=1)
    _, counts = np.unique(faces, axis=0, return_counts=True)
    assert counts.max() <= 2
    # the boundary faces tile the box surface: 2 triangles per boundary hex face
    nb = 2 * (n[0] * n[1] + n[1] * n[2] + n[0] * n[2])
    assert (counts == 1).sum() == 2 * nb


@pytest.mark.gpu
def test_reference_solid_test_scenario_on_the_gpu(block):
    """The reference's own solid test (tests/test_solid_bench.py:16-51) through this package:
    its mesh, Jacobi-PCG to rtol 1e-7 against the direct solve (<= 1e-6), non-negative von
    Mises; and against the reference's golden results on the same mesh: the direct solution
    (AMG-PCG to 1e-10, <= 1e-8) and the stress field of that solution (<= 1e-10)."""
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, compute_c3d10_stress_field, solve_c3d10_pcg

    g, m, meta = block
    K, F, fixed = assemble_c3d10_sparse_3dof(m)
    assert K.shape == (meta["n_dofs"], meta["n_dofs"]) and len(fixed) > 0
    assert np.array_equal(F, g["F"])
    u_pcg, iters, rel_res, _ = solve_c3d10_pcg(K, F, rtol=1e-7, preconditioner="jacobi")
    assert rel_res < 1e-7
    assert np.linalg.norm(g["u"] - u_pcg) <= 1e-6 * np.linalg.norm(g["u"])
    cell_sig, cell_vm, nodal_vm = compute_c3d10_stress_field(m, u_pcg)
    assert len(cell_sig) == meta["n_elements"] and np.all(cell_vm >= 0.0) and np.all(nodal_vm >= 0.0)
    assert nodal_vm.max() > 0.0
    u, _, rel, _ = solve_c3d10_pcg(K, F, rtol=1e-10, max_iter=2000, preconditioner="amg", precision="fp64")
    assert rel <= 1e-10
    assert np.linalg.norm(u - g["u"]) <= 1e-8 * np.linalg.norm(g["u"])
    _, vm, nvm = compute_c3d10_stress_field(m, g["u"])
    assert np.abs(vm - g["cell_vm"]).max() <= 1e-10 * g["cell_vm"].max()
    assert np.abs(nvm - g["nodal_vm"]).max() <= 1e-10 * g["nodal_vm"].max()
