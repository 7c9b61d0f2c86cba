"""Generate the golden fixtures of this directory by running the REFERENCE implementation.

Run in a container that has the reference checkout (read-only is fine):

    python tests/golden/make_golden.py /path/to/reference

The reference package does not import as shipped on Linux / Python 3.12 (wnfea/model.py:191
annotates with ``Path`` without importing it), so ``builtins.Path`` is set first.  Meshes
come from this repository's generators and are fed, as arrays, to the reference's own
functions, so both sides see identical inputs.  Fixtures:

* ``c3d10_element.npz``   -- element known answers from wnfea/elements/c3d10.py
                             (Ke of the scaled reference tet and a curved tet, f_int, stresses,
                             shape functions at the Gauss points);
* ``tiny_block.npz``      -- full K (apply_bcs False and True), F, fixed DOFs of a 2x1x1-hex
                             Kuhn block from assemble_c3d10_sparse_3dof (solid_solver.py:26-129);
* ``cantilever_c1.npz``   -- the 480-element cantilever: F, fixed, K @ v fingerprints, the
                             direct solution (spsolve), the reference Jacobi-PCG solution, and
                             the stress field (compute_c3d10_stress_field);
* ``beam_frame.npz``      -- the 10x10 co-rotational frame: F_int at a seeded displacement
                             from compute_internal_forces_fast's NumPy path
                             (fast_kernels.py:451-537) and the 10-step JFNK solution of
                             solve_nonlinear_jfnk (nonlinear_solver.py:159-376);
* ``structured_block.npz`` -- the reference's own mesh generator (generate_c3d10_structured_block,
                             solid_generator.py:21-213) with the arguments of its test
                             (tests/test_solid_bench.py:18-26): nodes, connectivity, clamped and
                             loaded nodes with their loads, and on that mesh the reference's
                             F, direct solution and stress field;
* ``bc_cases.npz``       -- the reference's assembly, direct solve and stresses on a model with
                             the boundary-condition cases its code distinguishes
                             (solid_solver.py:67-127): roller supports (one FIXED DOF per node on
                             three symmetry faces), a fully clamped corner, a duplicated support,
                             a PRESCRIBED DOF (not applied by the solid path), repeated loads on one
                             node, a load on a fixed DOF, two materials and elements left on the
                             default material.

    python tests/golden/make_golden.py /path/to/reference structured_block
    python tests/golden/make_golden.py /path/to/reference bc_cases

make only those.
"""

from __future__ import annotations

import builtins
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent


def structured_block(ref: str) -> None:
    builtins.Path = pathlib.Path
    sys.path.insert(0, ref)
    from scipy.sparse.linalg import spsolve
    from wnfea.mesh.solid_generator import generate_c3d10_structured_block
    from wnfea.solver.solid_solver import assemble_c3d10_sparse_3dof, compute_c3d10_stress_field

    model, meta = generate_c3d10_structured_block(length=5.0, width=1.0, height=1.0, nx=10, ny=3, nz=3,
                                                  tip_load_total=1000.0)
    K, F, fixed = assemble_c3d10_sparse_3dof(model)
    u = spsolve(K.tocsc(), F)
    cell_sig, cell_vm, nodal_vm = compute_c3d10_stress_field(model, u)
    np.savez_compressed(
        HERE / "structured_block.npz",
        nodes=np.asarray(model.mesh_nodes, dtype=np.float64),
        conn=np.asarray(model.solid_elements, dtype=np.int32),
        fixed_nodes=np.array([s.node_id for s in model.supports], dtype=np.int64),
        load_nodes=np.array([ld.node_id for ld in model.loads], dtype=np.int64),
        load_f=np.array([[ld.fx, ld.fy, ld.fz] for ld in model.loads], dtype=np.float64),
        counts=np.array([meta["n_nodes"], meta["n_elements"], meta["n_dofs"], meta["root_nodes_fixed"],
                         meta["tip_nodes_loaded"]], dtype=np.int64),
        F=F, fixed=np.asarray(fixed, dtype=np.int64), u=u, cell_sig=cell_sig, cell_vm=cell_vm, nodal_vm=nodal_vm)
    print("structured block", meta["n_elements"], "elements,", meta["n_dofs"], "DOFs")


def bc_case_model(wnfea, block):
    """The boundary-condition model on the mesh of ``block`` (a FEAModel of this repository),
    built with the reference's classes (and mirrored by tests/test_oracle_golden.py)."""
    from wnfea.boundary.conditions import DOFConstraint, DOFType, SupportDef

    X = block.mesh_nodes
    rm = wnfea.FEAModel()
    rm.mesh_nodes = X
    rm.solid_elements = block.solid_elements
    rm.materials["Steel"] = wnfea.MaterialDef("Steel", 2.1e11, 0.3, 2.5e8)
    rm.materials["Alu"] = wnfea.MaterialDef("Alu", 7.0e10, 0.33, 1.0e8)
    n_el = len(block.solid_elements)
    rm.solid_materials = {e: "Alu" for e in range(0, n_el, 3)}  # the rest: the default (first) material
    fixed = lambda: DOFConstraint(DOFType.FIXED)  # noqa: E731
    for axis, name in ((0, "ux"), (1, "uy"), (2, "uz")):
        for nid in np.flatnonzero(X[:, axis] <= 1e-12):
            rm.supports.append(SupportDef(node_id=int(nid), is_geometry_node=False, **{name: fixed()}))
    corner = int(np.argmin(np.abs(X - X.max(axis=0)).sum(axis=1)))
    rm.supports.append(wnfea.create_fixed_support(corner, is_geometry_node=False))
    rm.supports.append(wnfea.create_fixed_support(corner, is_geometry_node=False))  # duplicated
    mid = int(np.argmin(np.abs(X - 0.5 * X.max(axis=0)).sum(axis=1)))
    rm.supports.append(SupportDef(node_id=mid, is_geometry_node=False,
                                  uz=DOFConstraint(DOFType.PRESCRIBED, value=1e-3)))
    top = np.flatnonzero(X[:, 2] >= X[:, 2].max() - 1e-12)
    for k, nid in enumerate(top):
        rm.loads.append(wnfea.LoadDef(node_id=int(nid), is_geometry_node=False, fx=100.0 + k, fz=-500.0))
    rm.loads.append(wnfea.LoadDef(node_id=int(top[0]), is_geometry_node=False, fy=250.0))  # repeated node
    rm.loads.append(wnfea.LoadDef(node_id=corner, is_geometry_node=False, fx=1e6))  # on fixed DOFs
    return rm


def bc_cases(ref: str) -> None:
    builtins.Path = pathlib.Path
    sys.path.insert(0, ref)
    sys.path.insert(0, str(ROOT))
    import wnfea
    from scipy.sparse.linalg import spsolve
    from wnfea.solver.solid_solver import assemble_c3d10_sparse_3dof, compute_c3d10_stress_field

    from wnfea_b200.mesh import generate_c3d10_kuhn_block

    block, _ = generate_c3d10_kuhn_block(length=0.3, width=0.2, height=0.1, nx=3, ny=2, nz=2)
    rm = bc_case_model(wnfea, block)
    K, F, fixed = assemble_c3d10_sparse_3dof(rm)
    u = spsolve(K.tocsc(), F)
    cell_sig, cell_vm, nodal_vm = compute_c3d10_stress_field(rm, u)
    np.savez_compressed(HERE / "bc_cases.npz", nodes=block.mesh_nodes, conn=block.solid_elements,
                        K_data=K.data, K_indices=K.indices, K_indptr=K.indptr, F=F,
                        fixed=np.asarray(fixed, dtype=np.int64), u=u, cell_vm=cell_vm, nodal_vm=nodal_vm)
    print("bc cases", len(block.solid_elements), "elements,", len(fixed), "fixed DOFs")


def main(ref: str) -> None:
    builtins.Path = pathlib.Path
    sys.path.insert(0, ref)
    sys.path.insert(0, str(ROOT))
    import wnfea
    from scipy.sparse.linalg import spsolve
    from wnfea.elements import c3d10 as rc
    from wnfea.solver.solid_solver import (
        assemble_c3d10_sparse_3dof,
        compute_c3d10_stress_field,
        solve_c3d10_pcg,
    )

    from wnfea_b200.frames import generate_frame_grid
    from wnfea_b200.mesh import generate_c3d10_kuhn_block

    # ---- element known answers -------------------------------------------------------
    def ref_tet(scale):
        c = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64) * scale
        m = [0.5 * (c[a] + c[b]) for a, b in ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))]
        return np.vstack([c, np.array(m)])

    tet = ref_tet(1.5)
    curved = ref_tet(2.0)
    curved[4] += [0.02, 0.01, -0.01]
    curved[7] += [-0.01, 0.02, 0.01]
    rng = np.random.default_rng(99)
    u_e = rng.standard_normal(30) * 1e-3
    sig_gp, vm_gp, _ = rc.element_stresses_c3d10(curved, u_e, 2.0e11, 0.28)
    gps = np.array([np.asarray(g) for g in rc.GAUSS_POINTS_C3D10])
    N_gp = np.array([rc.shape_functions_c3d10(*g)[0] for g in gps])
    dN_gp = np.array([rc.shape_functions_c3d10(*g)[1] for g in gps])
    np.savez_compressed(
        HERE / "c3d10_element.npz",
        tet=tet,
        Ke_tet=rc.element_stiffness_c3d10(tet, 2.1e11, 0.3),
        curved=curved,
        Ke_curved=rc.element_stiffness_c3d10(curved, 1.8e11, 0.33),
        u_e=u_e,
        fint_curved=rc.element_internal_forces_c3d10(curved, u_e, 1.8e11, 0.33),
        sig_gp=sig_gp,
        vm_gp=vm_gp,
        gauss_points=gps,
        N_gp=N_gp,
        dN_gp=dN_gp,
    )

    def to_ref_model(m):
        rm = wnfea.FEAModel()
        rm.mesh_nodes = m.mesh_nodes
        rm.solid_elements = m.solid_elements
        for name, mat in m.materials.items():
            rm.materials[name] = wnfea.MaterialDef(name, mat.youngs_modulus, mat.poissons_ratio, mat.yield_strength)
        rm.solid_materials = {i: "Steel" for i in range(len(m.solid_elements))}
        for s in m.supports:
            rm.supports.append(wnfea.create_fixed_support(s.node_id, is_geometry_node=False))
        for ld in m.loads:
            rm.loads.append(wnfea.LoadDef(node_id=ld.node_id, is_geometry_node=False, fx=ld.fx, fy=ld.fy, fz=ld.fz))
        return rm

    # ---- tiny block: full matrices -------------------------------------------------------
    m, _ = generate_c3d10_kuhn_block(0.2, 0.1, 0.1, 2, 1, 1)
    rm = to_ref_model(m)
    K0, F0, _ = assemble_c3d10_sparse_3dof(rm, apply_bcs=False)
    K1, F1, fixed1 = assemble_c3d10_sparse_3dof(rm, apply_bcs=True)
    np.savez_compressed(
        HERE / "tiny_block.npz",
        nodes=m.mesh_nodes,
        conn=m.solid_elements,
        K0_data=K0.data, K0_indices=K0.indices, K0_indptr=K0.indptr,
        K1_data=K1.data, K1_indices=K1.indices, K1_indptr=K1.indptr,
        F=F1,
        fixed=np.asarray(fixed1, dtype=np.int64),
    )

    # ---- C1 cantilever -----------------------------------------------------------------
    m, _ = generate_c3d10_kuhn_block()
    rm = to_ref_model(m)
    K0, _, _ = assemble_c3d10_sparse_3dof(rm, apply_bcs=False)
    K, F, fixed = assemble_c3d10_sparse_3dof(rm, apply_bcs=True)
    v = np.random.default_rng(7).standard_normal(K.shape[0])
    u_direct = spsolve(K.tocsc(), F)
    t0 = time.perf_counter()
    u_pcg, iters, rel, _ = solve_c3d10_pcg(K, F, rtol=1e-10, max_iter=20000, preconditioner="jacobi")
    cell_sig, cell_vm, nodal_vm = compute_c3d10_stress_field(rm, u_direct)
    np.savez_compressed(
        HERE / "cantilever_c1.npz",
        nodes=m.mesh_nodes,
        conn=m.solid_elements,
        F=F,
        fixed=np.asarray(fixed, dtype=np.int64),
        K0_nnz=K0.nnz,
        K_nnz=K.nnz,
        K0_v=K0 @ v,
        K_v=K @ v,
        v=v,
        K_diag=K.diagonal(),
        u_direct=u_direct,
        u_pcg=u_pcg,
        pcg_rel=rel,
        cell_sig=cell_sig,
        cell_vm=cell_vm,
        nodal_vm=nodal_vm,
    )
    print("C1: K nnz", K.nnz, "tip uz", u_direct.reshape(-1, 3)[:, 2].min(), "pcg", time.perf_counter() - t0)

    # ---- co-rotational beam frame ------------------------------------------------------
    from wnfea.solver.fast_kernels import compute_internal_forces_fast
    from wnfea.solver.nonlinear_solver import solve_nonlinear_jfnk

    fm = generate_frame_grid()
    rfm = wnfea.FEAModel()
    rfm.mesh_nodes = fm.mesh_nodes
    rfm.mesh_elements = fm.mesh_elements
    for name, mat in fm.materials.items():
        rfm.materials[name] = wnfea.MaterialDef(name, mat.youngs_modulus, mat.poissons_ratio, mat.yield_strength)
    for name, sec in fm.sections.items():
        rfm.sections[name] = wnfea.SectionDef(name, sec.area, sec.iy, sec.iz, sec.j)
    for eid, a in fm.element_properties.items():
        rfm.element_properties[eid] = wnfea.PropertyAssignment(a.material_name, a.section_name)
    for s in fm.supports:
        rfm.supports.append(wnfea.create_fixed_support(s.node_id, is_geometry_node=False))
    for ld in fm.loads:
        rfm.loads.append(wnfea.LoadDef(node_id=ld.node_id, is_geometry_node=False, fz=ld.fz))
    U = np.random.default_rng(11).standard_normal(len(fm.mesh_nodes) * 6) * 1e-3
    fint = compute_internal_forces_fast(rfm, U.copy(), device="cpu")
    rfm._batch_data = None
    t0 = time.perf_counter()
    U_nl = solve_nonlinear_jfnk(rfm, n_load_steps=10, tol_rel=1e-12, tol_abs=1e-5, verbose=False)
    print("frame JFNK", time.perf_counter() - t0, "max |uz|", np.abs(U_nl.reshape(-1, 6)[:, 2]).max())
    np.savez_compressed(HERE / "beam_frame.npz", U=U, fint=fint, U_nl=U_nl)


if __name__ == "__main__":
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    if len(sys.argv) > 2 and sys.argv[2] == "structured_block":
        structured_block(ref_dir)
    elif len(sys.argv) > 2 and sys.argv[2] == "bc_cases":
        bc_cases(ref_dir)
    else:
        main(ref_dir)
        structured_block(ref_dir)
        bc_cases(ref_dir)
