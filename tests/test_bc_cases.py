"""Boundary-condition cases of the solid path against the reference's own results.

tests/golden/bc_cases.npz holds what the reference's assemble_c3d10_sparse_3dof, spsolve and
compute_c3d10_stress_field (solid_solver.py:26-129, 311-365) return for a model with every case
its code distinguishes: roller supports (one FIXED DOF per node on three symmetry faces), a fully
clamped corner listed twice, a PRESCRIBED DOF (the solid path applies only FIXED ones), repeated
loads on one node, a load on fixed DOFs (zeroed), two materials and elements left on the default
(first) material.  The model is rebuilt here with this package's classes, as a caller would.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import solid
from wnfea_b200.mesh import generate_c3d10_kuhn_block
from wnfea_b200.model import (DOFConstraint, DOFType, FEAModel, LoadDef, MaterialDef, SupportDef,
                              create_fixed_support, solid_element_props, solid_fixed_dofs, solid_load_vector)

GOLDEN = Path(__file__).resolve().parent / "golden" / "bc_cases.npz"


def bc_model():
    """The model of tests/golden/make_golden.py bc_case_model, with this package's classes."""
    block, _ = generate_c3d10_kuhn_block(length=0.3, width=0.2, height=0.1, nx=3, ny=2, nz=2)
    X = block.mesh_nodes
    m = FEAModel()
    m.mesh_nodes = X
    m.solid_elements = block.solid_elements
    m.materials["Steel"] = MaterialDef("Steel", 2.1e11, 0.3, 2.5e8)
    m.materials["Alu"] = MaterialDef("Alu", 7.0e10, 0.33, 1.0e8)
    m.solid_materials = {e: "Alu" for e in range(0, len(block.solid_elements), 3)}
    for axis, name in ((0, "ux"), (1, "uy"), (2, "uz")):
        for nid in np.flatnonzero(X[:, axis] <= 1e-12):
            m.supports.append(SupportDef(node_id=int(nid), is_geometry_node=False,
                                         **{name: DOFConstraint(DOFType.FIXED)}))
    corner = int(np.argmin(np.abs(X - X.max(axis=0)).sum(axis=1)))
    m.supports.append(create_fixed_support(corner, is_geometry_node=False))
    m.supports.append(create_fixed_support(corner, is_geometry_node=False))
    mid = int(np.argmin(np.abs(X - 0.5 * X.max(axis=0)).sum(axis=1)))
    m.supports.append(SupportDef(node_id=mid, is_geometry_node=False, uz=DOFConstraint(DOFType.PRESCRIBED, value=1e-3)))
    top = np.flatnonzero(X[:, 2] >= X[:, 2].max() - 1e-12)
    for k, nid in enumerate(top):
        m.loads.append(LoadDef(node_id=int(nid), is_geometry_node=False, fx=100.0 + k, fz=-500.0))
    m.loads.append(LoadDef(node_id=int(top[0]), is_geometry_node=False, fy=250.0))
    m.loads.append(LoadDef(node_id=corner, is_geometry_node=False, fx=1e6))
    return m


@pytest.fixture(scope="module")
def golden():
    g = np.load(GOLDEN)
    n = len(g["F"])
    K = sp.csr_matrix((g["K_data"], g["K_indices"], g["K_indptr"]), shape=(n, n))
    return g, K


def test_bc_cases_oracle_matches_reference(golden):
    g, Kr = golden
    m = bc_model()
    assert np.array_equal(m.mesh_nodes, g["nodes"]) and np.array_equal(m.solid_elements, g["conn"])
    assert np.array_equal(solid_fixed_dofs(m), g["fixed"])  # support order, duplicates kept
    F = solid_load_vector(m)
    F[np.asarray(solid_fixed_dofs(m))] = 0.0
    assert np.array_equal(F, g["F"])
    Ko, Fo, fixed = solid.assemble(m.mesh_nodes, m.solid_elements, solid_element_props(m), solid_load_vector(m),
                                   solid_fixed_dofs(m))
    assert np.array_equal(Fo, g["F"])
    assert abs(Ko - Kr).max() <= 1e-14 * abs(Kr).max()


@pytest.mark.gpu
def test_bc_cases_gpu_matches_reference(golden):
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, compute_c3d10_stress_field, solve_c3d10_pcg

    g, Kr = golden
    m = bc_model()
    K, F, fixed = assemble_c3d10_sparse_3dof(m)
    assert np.array_equal(np.asarray(fixed), g["fixed"])
    assert np.array_equal(F, g["F"])
    assert abs(K.tocsr() - Kr).max() <= 1e-14 * abs(Kr).max()
    fx = np.asarray(fixed)
    for precond in ("amg", "jacobi", "block_jacobi"):
        u, _, rel, _ = solve_c3d10_pcg(K, F, rtol=1e-10, max_iter=20000, preconditioner=precond, precision="fp64")
        assert rel <= 1e-10, precond
        assert np.linalg.norm(u - g["u"]) <= 1e-8 * np.linalg.norm(g["u"]), precond
        # fixed DOFs: identity rows with zero load, decoupled in the AMG and point-Jacobi
        # preconditioners (exact zeros); the 3x3 block pseudo-inverses of roller nodes, from an
        # eigen-decomposition, may couple them at rounding level
        if precond == "block_jacobi":
            assert np.abs(u[fx]).max() <= 1e-12 * np.abs(u).max()
        else:
            assert np.all(u[fx] == 0.0), precond
    _, vm, nvm = compute_c3d10_stress_field(m, g["u"])
    assert np.abs(vm - g["cell_vm"]).max() <= 1e-10 * g["cell_vm"].max()
    assert np.abs(nvm - g["nodal_vm"]).max() <= 1e-10 * g["nodal_vm"].max()
