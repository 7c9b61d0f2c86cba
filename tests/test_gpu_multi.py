"""Multi-right-hand-side PCG (32 load cases per batch) on the GPU: every case against a direct
solve of the oracle's matrix, against the single-case GPU solve, and through properties that
hold exactly for independent per-case recurrences (scaling by 2, independence of the other
cases in the batch, graph replay, determinism)."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.sparse.linalg import splu

from oracle import solid
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block, tip_load_cases
from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector
from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_multi

pytestmark = pytest.mark.gpu


def _ibeam(n_slices=12, seed=5):
    m, _ = generate_c3d10_ibeam_structured(n_slices=n_slices, length=4.0 * n_slices / 315, seed=seed)
    return m


def _direct(m, F):
    K, _, _ = solid.assemble(m.mesh_nodes, m.solid_elements, solid_element_props(m), solid_load_vector(m),
                             solid_fixed_dofs(m))
    lu = splu(K.tocsc())
    return lu.solve(F)


@pytest.mark.parametrize("precision,rtol,tol", [("fp64", 1e-10, 1e-8), ("mixed_fp32", 1e-8, 1e-6)])
def test_cases_match_direct_solve(precision, rtol, tol):
    """40 cases = one full batch of 32 and a padded batch of 8."""
    m, _ = generate_c3d10_kuhn_block()
    K, _, _ = assemble_c3d10_sparse_3dof(m)
    F = tip_load_cases(m.mesh_nodes, n_cases=40, seed=1)
    U, st = solve_c3d10_multi(K, F, rtol=rtol, precision=precision)
    assert st["status"] == 0
    assert (st["case_rel_res"] <= rtol).all() and st["rel_res"] <= rtol
    assert (st["case_iterations"] > 0).all()
    Ur = _direct(m, F)
    err = np.linalg.norm(U - Ur, axis=0) / np.linalg.norm(Ur, axis=0)
    assert err.max() < tol, err.max()


def test_case_iterations_track_single_case_solves():
    m = _ibeam(10, seed=2)
    K, _, _ = assemble_c3d10_sparse_3dof(m)
    F = tip_load_cases(m.mesh_nodes, n_cases=6, seed=3)
    s = K.system
    s.amg_setup()
    U, st = s.solve_multi(F, rtol=1e-8, precision=1)
    for j in range(F.shape[1]):
        u, sj = s.solve(F[:, j], rtol=1e-8, precision=1)
        assert abs(int(st["case_iterations"][j]) - sj["iterations"]) <= max(2, 0.1 * sj["iterations"])
        assert np.linalg.norm(U[:, j] - u) <= 1e-6 * np.linalg.norm(u)


def test_exact_case_properties():
    """Per-case recurrences: a case scaled by 2 gives exactly twice the solution, and a
    case's result does not depend on the other cases of its batch."""
    m = _ibeam(8, seed=4)
    K, _, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    s.amg_setup()
    F = tip_load_cases(m.mesh_nodes, n_cases=5, seed=6)
    F2 = np.column_stack([F, 2.0 * F[:, 1]])
    for precision in (0, 1):
        U, st = s.solve_multi(F2, rtol=1e-9, precision=precision)
        assert np.array_equal(U[:, 5], 2.0 * U[:, 1])
        assert st["case_iterations"][5] == st["case_iterations"][1]
        U1, _ = s.solve_multi(F[:, 3:4], rtol=1e-9, precision=precision)
        assert np.array_equal(U1[:, 0], U[:, 3])
        # CUDA-graph replay and direct launches give identical bits; so does a second run
        Ua, _ = s.solve_multi(F, rtol=1e-9, precision=precision, use_graph=False, chunk=4)
        Ub, _ = s.solve_multi(F, rtol=1e-9, precision=precision, use_graph=True, chunk=4)
        Uc, _ = s.solve_multi(F, rtol=1e-9, precision=precision, use_graph=True, chunk=4)
        assert np.array_equal(Ua, Ub) and np.array_equal(Ub, Uc)


def test_zero_and_corrupt_cases():
    m, _ = generate_c3d10_kuhn_block()
    K, _, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    F = tip_load_cases(m.mesh_nodes, n_cases=4, seed=2)
    F[:, 0] = 0.0
    U, st = s.solve_multi(F, rtol=1e-8, precision=1)
    assert st["status"] == 0 and not U[:, 0].any() and st["case_iterations"][0] == 0
    Fn = F.copy()
    Fn[7, 2] = np.nan  # reported as a breakdown of that case; the others still converge
    Un, stn = s.solve_multi(Fn, rtol=1e-8, precision=1)
    assert stn["status"] == -4
    good = [1, 3]
    assert (stn["case_rel_res"][good] <= 1e-8).all()
    assert np.array_equal(Un[:, good], U[:, good])
    # iteration limit
    _, stl = s.solve_multi(F, rtol=1e-14, max_iter=3, precision=1, max_outer=1)
    assert stl["status"] == -5 and stl["iterations"] == 3


def test_ibeam_mixed_batch_matches_fp64():
    m = _ibeam(16, seed=7)
    K, _, _ = assemble_c3d10_sparse_3dof(m)
    F = tip_load_cases(m.mesh_nodes, n_cases=32, seed=0)
    U64, st64 = solve_c3d10_multi(K, F, rtol=1e-10, precision="fp64")
    U32, st32 = solve_c3d10_multi(K, F, rtol=1e-8, precision="mixed_fp32")
    assert st64["status"] == 0 and st32["status"] == 0
    Ur = _direct(m, F)
    e64 = np.linalg.norm(U64 - Ur, axis=0) / np.linalg.norm(Ur, axis=0)
    e32 = np.linalg.norm(U32 - Ur, axis=0) / np.linalg.norm(Ur, axis=0)
    assert e64.max() < 1e-8 and e32.max() < 1e-6


def test_streamed_fine_level_matches_register_kernels():
    """The batched fine level on its three paths: the register row kernels (the default), x
    staged per row tile in shared memory (staging on) and streamed from the tile-major pack
    (streaming mode 2).  Each runs the same per-case arithmetic in the same order, so the row
    products agree bit for bit and the solves differ only by the order in which the per-CTA dot
    partials are summed.  Switching paths between solves re-captures the batched solver's
    graphs (streaming off frees the packs, mode 2 rebuilds them), and returning to the default
    reproduces its first result exactly."""
    from wnfea_b200 import _lib

    m = _ibeam(20, seed=8)
    K, _, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    s.amg_setup()
    F = tip_load_cases(m.mesh_nodes, n_cases=32, seed=4)
    F[np.asarray(solid_fixed_dofs(m), dtype=np.int64), :] = 0.0
    for precision in (0, 1):
        U1, st1 = s.solve_multi(F, rtol=1e-9, precision=precision)
        try:
            _lib.call("wn_solid_set_stream", s.handle, 2)
            U2, st2 = s.solve_multi(F, rtol=1e-9, precision=precision)
            _lib.call("wn_solid_set_stream", s.handle, 0)
            U0, st0 = s.solve_multi(F, rtol=1e-9, precision=precision)
            _lib.call("wn_solid_set_batch_staging", s.handle, 1)
            Ur, str_ = s.solve_multi(F, rtol=1e-9, precision=precision)
        finally:
            _lib.call("wn_solid_set_batch_staging", s.handle, 0)
            _lib.call("wn_solid_set_stream", s.handle, 1)
        U1b, st1b = s.solve_multi(F, rtol=1e-9, precision=precision)
        for st in (st0, st1, st2, str_, st1b):
            assert st["status"] == 0
        assert np.array_equal(U1, U1b)
        for U, st in ((U2, st2), (U0, st0), (Ur, str_)):
            assert np.abs(st["case_iterations"] - st1["case_iterations"]).max() <= 1
            assert np.linalg.norm(U - U1) <= 1e-9 * np.linalg.norm(U1)
