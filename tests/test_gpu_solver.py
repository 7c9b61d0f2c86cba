"""GPU parity of the AMG V-cycle and the PCG / mixed-precision solver (through the C ABI)
against the oracle restatement, scipy and the reference's golden solution."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import spsolve

from oracle import amg as oamg
from oracle import solid
from wnfea_b200 import _lib
from wnfea_b200.amg import AMGParams, export_system_hierarchy
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block
from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector
from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_pcg, solve_c3d10_system
from wnfea_b200.system import SolidSystem

pytestmark = pytest.mark.gpu


def _ibeam(n_slices=16, seed=3):
    m, _ = generate_c3d10_ibeam_structured(n_slices=n_slices, length=4.0 * n_slices / 315, seed=seed)
    return m


def _oracle_K(m):
    K, F, _ = solid.assemble(m.mesh_nodes, m.solid_elements, solid_element_props(m), solid_load_vector(m),
                             solid_fixed_dofs(m))
    return K, F


@pytest.mark.parametrize("which", ["c1", "ibeam"])
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_vcycle_matches_oracle(which, degree):
    import torch

    m = generate_c3d10_kuhn_block()[0] if which == "c1" else _ibeam()
    K, F, fixed = assemble_c3d10_sparse_3dof(m)
    s = K.system
    prm = AMGParams(coarse_size=300, smoother_degree=degree, cheb_lower=1.0 / 16.0 if degree == 1 else 1.0 / 30.0)
    s.amg_setup(prm)
    H = export_system_hierarchy(s)
    Kfull = K.to_bsr().tocsr()  # with explicit zeros, as the GPU sees it
    r = np.random.default_rng(1).standard_normal(K.shape[0])
    z_ref = oamg.vcycle(Kfull, H, r, degree=degree, lower=prm.cheb_lower, safety=prm.cheb_safety)
    dr = torch.from_numpy(r).cuda()
    dz = torch.empty_like(dr)
    _lib.call("wn_amg_vcycle_device", s.handle, 0, dr.data_ptr(), dz.data_ptr(), 0)
    torch.cuda.synchronize()
    z = dz.cpu().numpy()
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) < 1e-10
    dr32 = dr.float()
    dz32 = torch.empty_like(dr32)
    _lib.call("wn_amg_vcycle_device", s.handle, 1, dr32.data_ptr(), dz32.data_ptr(), 0)
    torch.cuda.synchronize()
    z32 = dz32.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(z32 - z_ref) / np.linalg.norm(z_ref) < 1e-4
    # symmetric positive definite preconditioner (test_nonlinear_jfnk.py:108-114)
    assert r @ z > 0


def test_fp64_amg_solution_matches_reference(golden):
    g = golden("cantilever_c1.npz")
    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    # the true FP64 residual floors near ||K|| ||u|| eps / ||F|| (about 1e-10 here), and the
    # solver stops on the true residual
    u, st = solve_c3d10_system(K, F, method="pcg", rtol=3e-10, preconditioner="amg", precision="fp64")
    assert st["status"] == 0 and st["rel_res"] < 3e-10
    rel = np.linalg.norm(u - g["u_direct"]) / np.linalg.norm(g["u_direct"])
    assert rel < 1e-8, rel
    u8, st8 = solve_c3d10_system(K, F, method="pcg", rtol=1e-8, preconditioner="amg", precision="fp64")
    assert st8["rel_res"] < 1e-8
    assert np.linalg.norm(u8 - g["u_direct"]) / np.linalg.norm(g["u_direct"]) < 1e-6


def test_mixed_solution_matches_reference(golden):
    g = golden("cantilever_c1.npz")
    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    u, st = solve_c3d10_system(K, F, method="pcg", rtol=1e-8, preconditioner="amg", precision="mixed_fp32")
    assert st["status"] == 0 and st["rel_res"] < 1e-8 and st["outer_iters"] >= 1
    rel = np.linalg.norm(u - g["u_direct"]) / np.linalg.norm(g["u_direct"])
    assert rel < 1e-6, rel


def test_jacobi_pcg_matches_reference_iterations():
    """Point-Jacobi PCG: same algorithm as the reference's default (scipy cg + Jacobi)."""
    import scipy.sparse.linalg as spla

    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    Ko, Fo = _oracle_K(m)
    # The GPU solver asks its PCG for 0.5 rtol and then checks the true FP64 residual, adding
    # a short refinement pass if the recursive residual drifted; scipy stops on its recursive
    # residual.  Compare the first pass at the same target, then the full solve.
    _, its_ref, rel_ref, _ = solid.pcg(Ko, Fo, rtol=0.5e-8, max_iter=5000)
    _, st1 = K.system.solve(F, rtol=1e-8, max_iter=5000, precond=1, max_outer=1)
    assert st1["outer_iterations"] == 1
    its = st1["iterations"]
    # same recurrence; over ~750 iterations of this ill-conditioned system the FP64 rounding
    # of the dot products (fixed-order block sums here, pairwise sums in numpy) moves the
    # count by a few percent
    assert abs(its - its_ref) <= 0.06 * its_ref + 3, (its, its_ref)
    u, its_all, rel, _ = solve_c3d10_pcg(K, F, rtol=1e-8, max_iter=5000, preconditioner="jacobi")
    assert rel <= 1e-8
    u_ref = spsolve(Ko.tocsc(), Fo)
    assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) < 1e-6


def test_block_jacobi_pcg_matches_reference_iterations():
    """3x3 block-Jacobi PCG (pseudo-inverse of every node block, solid_solver.py:237-258)."""
    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    Ko, Fo = _oracle_K(m)
    _, its_ref, _, _ = solid.pcg(Ko, Fo, rtol=0.5e-8, max_iter=5000, preconditioner="block_jacobi")
    _, its_pt, _, _ = solid.pcg(Ko, Fo, rtol=0.5e-8, max_iter=5000, preconditioner="jacobi")
    assert its_ref != its_pt  # the two preconditioners are told apart by their counts
    _, st1 = K.system.solve(F, rtol=1e-8, max_iter=5000, precond=3, max_outer=1)
    assert st1["outer_iterations"] == 1
    its = st1["iterations"]
    assert abs(its - its_ref) <= 0.06 * its_ref + 3, (its, its_ref)
    u_ref = spsolve(Ko.tocsc(), Fo)
    for precision, tol in (("fp64", 1e-6), ("mixed_fp32", 1e-6)):
        u, its_all, rel, _ = solve_c3d10_pcg(K, F, rtol=1e-8, max_iter=5000, preconditioner="block_jacobi",
                                             precision=precision)
        assert rel <= 1e-8, (precision, rel)
        assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) < tol, precision


def test_reference_default_preconditioner_is_jacobi():
    """solve_c3d10_pcg / solve_c3d10_system keep the reference's defaults (point Jacobi, rtol
    1e-6, 2000 iterations, FP64): the default call runs the Jacobi recurrence."""
    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    _, its_default, rel_default, _ = solve_c3d10_pcg(K, F)
    _, its_jac, rel_jac, _ = solve_c3d10_pcg(K, F, preconditioner="jacobi")
    assert its_default == its_jac and rel_default == rel_jac
    _, st = solve_c3d10_system(K, F, method="pcg")
    assert st["method"] == "pcg_jacobi_fp64" and st["iterations"] == its_jac


def test_ibeam_fp64_and_mixed_agree():
    m = _ibeam(24, seed=7)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    Ko, Fo = _oracle_K(m)
    u_ref = spsolve(Ko.tocsc(), Fo)
    u64, st64 = solve_c3d10_system(K, F, method="pcg", rtol=1e-10, preconditioner="amg", precision="fp64")
    u32, st32 = solve_c3d10_system(K, F, method="pcg", rtol=1e-8, preconditioner="amg", precision="mixed_fp32")
    assert st64["status"] == 0 and st32["status"] == 0
    assert np.linalg.norm(u64 - u_ref) / np.linalg.norm(u_ref) < 1e-8
    assert np.linalg.norm(u32 - u_ref) / np.linalg.norm(u_ref) < 1e-6
    assert st32["rel_res"] < 1e-8


def test_graph_replay_is_bit_identical_to_direct_launches():
    m = _ibeam(10, seed=2)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    s.amg_setup()
    for precision in (0, 1):
        ua, sa = s.solve(F, rtol=1e-9, precision=precision, use_graph=True, chunk=4)
        ub, sb = s.solve(F, rtol=1e-9, precision=precision, use_graph=False, chunk=4)
        uc, sc = s.solve(F, rtol=1e-9, precision=precision, use_graph=True, chunk=4)
        assert np.array_equal(ua, ub) and np.array_equal(ua, uc)
        assert sa["iterations"] == sb["iterations"] == sc["iterations"]


def test_zero_rhs_and_iteration_limit_and_nan():
    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    u, st = s.solve(np.zeros_like(F), rtol=1e-8)
    assert st["status"] == 0 and st["iterations"] == 0 and not u.any()
    u, st = s.solve(F, rtol=1e-14, max_iter=3, precond=1)
    assert st["status"] == -5 and st["iterations"] == 3  # WN_ENOCONV, bounded by max_iter
    Fn = F.copy()
    Fn[5] = np.nan  # a corrupted load vector is reported, not iterated on
    u, st = s.solve(Fn, rtol=1e-8)
    assert st["status"] == -4  # WN_EBREAKDOWN


def test_solve_is_deterministic():
    m = _ibeam(8, seed=4)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    u1, _ = solve_c3d10_system(K, F, method="pcg", rtol=1e-9, preconditioner="amg", precision="mixed_fp32")
    u2, _ = solve_c3d10_system(K, F, method="pcg", rtol=1e-9, preconditioner="amg", precision="mixed_fp32")
    assert np.array_equal(u1, u2)


def test_fp32_iterative_refinement_mode_on_small_mesh(golden):
    """The reference's mixed mode (FP32 PCG inside FP64 refinement) on the 480-element case."""
    g = golden("cantilever_c1.npz")
    m, _ = generate_c3d10_kuhn_block()
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    u, st = solve_c3d10_system(K, F, method="pcg", rtol=1e-8, preconditioner="amg", precision="mixed_fp32_ir")
    assert st["status"] == 0 and st["rel_res"] < 1e-8 and st["outer_iters"] >= 2
    assert np.linalg.norm(u - g["u_direct"]) / np.linalg.norm(g["u_direct"]) < 1e-6


def _residual_longdouble(K, u, F):
    """(||F - K u|| / ||F||, eps64 || |K| |u| || / ||F||) with the products and sums in extended
    precision (x86 80-bit): the residual of the FP64 vector u, resolved below the FP64 rounding
    level of K u, and that rounding level (no FP64 vector has a residual much below it)."""
    Kc = K.tocsr()
    uu = u.astype(np.longdouble)[Kc.indices]
    prod = Kc.data.astype(np.longdouble) * uu
    Ku = np.add.reduceat(prod, Kc.indptr[:-1])
    aKu = np.add.reduceat(np.abs(prod), Kc.indptr[:-1])
    r = F.astype(np.longdouble) - Ku
    fn = np.sqrt((F.astype(np.longdouble) ** 2).sum())
    return float(np.sqrt((r * r).sum()) / fn), float(np.finfo(np.float64).eps * np.sqrt((aKu * aKu).sum()) / fn)


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("mixed_fp32", 1e-10)])
def test_tight_tolerance_on_lateral_load(precision, rtol):
    """A weak-axis (lateral) tip load: large displacements put the FP64 rounding level of K u
    near the requested residual.  The refined (double-double) solution reaches rtol; the FP64
    vector returned is its rounding, whose residual is at rtol or at the FP64 rounding level."""
    m = _ibeam(40, seed=1)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    Ko, Fo = _oracle_K(m)
    tip = np.flatnonzero(m.mesh_nodes[:, 0] >= m.mesh_nodes[:, 0].max() - 1e-12)
    Fy = np.zeros_like(F)
    Fy[3 * tip + 1] = 50e3 / len(tip)
    u, st = solve_c3d10_system(K, Fy, method="pcg", rtol=rtol, preconditioner="amg", precision=precision, max_iter=4000)
    assert st["status"] == 0 and st["rel_res"] <= rtol
    res, floor = _residual_longdouble(Ko, u, Fy)
    assert res <= 2 * max(rtol, floor)


def test_tiny_mesh_hierarchy_without_levels():
    """Fewer DOFs than the coarse-solve size: the 'V-cycle' is the dense coarse solve alone."""
    from wnfea_b200.mesh import tip_load_cases

    m, _ = generate_c3d10_kuhn_block(length=0.2, width=0.1, height=0.1, nx=2, ny=2, nz=2)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    Ko, Fo = _oracle_K(m)
    ur = spsolve(Ko.tocsc(), Fo)
    for precision in ("fp64", "mixed_fp32"):
        u, st = solve_c3d10_system(K, F, method="pcg", rtol=1e-10, preconditioner="amg", precision=precision)
        assert st["status"] == 0 and st["levels"] == 1
        assert np.linalg.norm(u - ur) <= 1e-8 * np.linalg.norm(ur)
    Fm = tip_load_cases(m.mesh_nodes, n_cases=3, seed=0)
    U, stm = K.system.solve_multi(Fm, rtol=1e-10, precision=1)
    assert stm["status"] == 0
    Ur = spsolve(Ko.tocsc(), Fm)
    assert np.linalg.norm(U - Ur) <= 1e-8 * np.linalg.norm(Ur)


def test_profiled_solve_accounts_every_kernel():
    """params.profile: the same solve with an event after every kernel.  The solution is bitwise
    the normal one; the per-class algorithmic bytes add up to the solve's algorithmic_bytes (the
    classes count exactly the launches that did their work); the classes name the V-cycle stages
    per level, the PCG kernels and the outer-residual kernels."""
    m = _ibeam(12, seed=4)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    for degree, precision in ((1, 0), (1, 1), (2, 0), (2, 1)):
        s.amg_setup(AMGParams(smoother_degree=degree))
        u0, st0 = s.solve(F, rtol=1e-8, precision=precision)
        u1, st1 = s.solve(F, rtol=1e-8, precision=precision, profile=True)
        assert st0["status"] == 0 and st1["status"] == 0
        assert np.array_equal(u0, u1) and st0["iterations"] == st1["iterations"]
        assert st0["algorithmic_bytes"] > 0 and abs(st1["algorithmic_bytes"] - st0["algorithmic_bytes"]) <= (
            1e-12 * st0["algorithmic_bytes"])
        prof = s.profile_table()
        names = ["pcg_spmv_dot", "pcg_update", "l0.pre_smooth", "l0.restrict", "l0.prolong", "l0.post_smooth", "coarse",
                 "outer_residual"]
        if degree >= 2:  # the residual after the pre-smoother and the second post-smoothing step
            names += ["l0.residual", "l0.post_cheb"]
        else:
            assert "l0.residual" not in prof and "l0.post_cheb" not in prof
        for name in names:
            assert name in prof, (name, sorted(prof))
        its = st1["iterations"]
        assert prof["pcg_spmv_dot"][0] == its and prof["pcg_update"][0] == its
        assert prof["coarse"][0] == its  # the initial apply plus one per iteration but the last
        total = sum(v[2] for v in prof.values())
        assert abs(total - st1["algorithmic_bytes"]) <= 1e-9 * total
        assert 0 < sum(v[1] for v in prof.values()) <= st1["solve_seconds"] * 1e3 * 1.01
