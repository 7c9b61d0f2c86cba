"""The oracle pinned against golden vectors produced by the reference itself (CPU only)."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import beam, c3d10, solid
from wnfea_b200.frames import generate_frame_grid


def test_shape_functions_match_reference(golden):
    g = golden("c3d10_element.npz")
    for k, gp in enumerate(g["gauss_points"]):
        N, dN = c3d10.shape_functions(*gp)
        np.testing.assert_allclose(N, g["N_gp"][k], rtol=0, atol=1e-15)
        np.testing.assert_allclose(dN, g["dN_gp"][k], rtol=0, atol=1e-14)


def test_partition_of_unity_and_kronecker():
    # test_c3d10.py:46-81
    nat = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (0.5, 0, 0), (0.5, 0.5, 0), (0, 0.5, 0), (0, 0, 0.5),
           (0.5, 0, 0.5), (0, 0.5, 0.5)]
    for j, p in enumerate(nat):
        N, _ = c3d10.shape_functions(*p)
        np.testing.assert_allclose(N, np.eye(10)[j], atol=1e-14)
    rng = np.random.default_rng(42)
    for _ in range(20):
        r = rng.dirichlet(np.ones(4))
        N, dN = c3d10.shape_functions(r[1], r[2], r[3])
        assert abs(N.sum() - 1) < 1e-14
        np.testing.assert_allclose(dN.sum(axis=1), 0, atol=1e-14)


def test_element_stiffness_matches_reference(golden):
    g = golden("c3d10_element.npz")
    Ke = c3d10.element_stiffness_batch(g["tet"][None], np.array([[2.1e11, 0.3]]))[0]
    np.testing.assert_allclose(Ke, g["Ke_tet"], rtol=0, atol=1e-14 * np.abs(g["Ke_tet"]).max())
    Ke = c3d10.element_stiffness_batch(g["curved"][None], np.array([[1.8e11, 0.33]]))[0]
    np.testing.assert_allclose(Ke, g["Ke_curved"], rtol=0, atol=1e-14 * np.abs(g["Ke_curved"]).max())


def test_element_force_and_stress_match_reference(golden):
    g = golden("c3d10_element.npz")
    f = c3d10.element_internal_forces_batch(g["curved"][None], g["u_e"][None], np.array([[1.8e11, 0.33]]))[0]
    np.testing.assert_allclose(f, g["fint_curved"], rtol=0, atol=1e-13 * np.abs(f).max())
    sig, vm = c3d10.element_stresses_batch(g["curved"][None], g["u_e"][None], np.array([[2.0e11, 0.28]]))
    np.testing.assert_allclose(sig[0], g["sig_gp"], rtol=1e-12, atol=1e-6)
    np.testing.assert_allclose(vm[0], g["vm_gp"], rtol=1e-12)


def _csr(g, p):
    n = len(g[p + "_indptr"]) - 1
    return sp.csr_matrix((g[p + "_data"], g[p + "_indices"], g[p + "_indptr"]), shape=(n, n))


def test_assembly_matches_reference_tiny(golden):
    g = golden("tiny_block.npz")
    props = np.tile([2.1e11, 0.3], (len(g["conn"]), 1))
    n = 3 * len(g["nodes"])
    F = np.zeros(n)
    K0, _, _ = solid.assemble(g["nodes"], g["conn"], props, F, g["fixed"], apply_bcs=False)
    R0 = _csr(g, "K0")
    assert (K0.indptr == R0.indptr).all() and (K0.indices == R0.indices).all()
    np.testing.assert_allclose(K0.toarray(), R0.toarray(), rtol=0, atol=1e-14 * abs(R0).max())
    K1, F1, fixed = solid.assemble(g["nodes"], g["conn"], props, F, g["fixed"], apply_bcs=True)
    R1 = _csr(g, "K1")
    np.testing.assert_allclose(K1.toarray(), R1.toarray(), rtol=0, atol=1e-14 * abs(R1).max())
    assert list(fixed) == list(g["fixed"])


def test_cantilever_fingerprints_and_solution(golden):
    g = golden("cantilever_c1.npz")
    props = np.tile([2.1e11, 0.3], (len(g["conn"]), 1))
    K0, _, _ = solid.assemble(g["nodes"], g["conn"], props, g["F"], g["fixed"], apply_bcs=False)
    assert K0.nnz == int(g["K0_nnz"])
    np.testing.assert_allclose(K0 @ g["v"], g["K0_v"], rtol=0, atol=1e-13 * np.abs(g["K0_v"]).max())
    K, F, _ = solid.assemble(g["nodes"], g["conn"], props, g["F"], g["fixed"], apply_bcs=True)
    np.testing.assert_allclose(K @ g["v"], g["K_v"], rtol=0, atol=1e-13 * np.abs(g["K_v"]).max())
    np.testing.assert_allclose(F, g["F"], rtol=0, atol=0)
    u, its, rel, _ = solid.pcg(K, F, rtol=1e-10, max_iter=20000)
    assert rel < 1e-9  # scipy cg stops on its recursive residual; the true one trails it
    np.testing.assert_allclose(u, g["u_direct"], rtol=0, atol=1e-7 * np.abs(g["u_direct"]).max())
    sig, vm, nvm = solid.stress_field(g["nodes"], g["conn"], props, g["u_direct"])
    np.testing.assert_allclose(sig, g["cell_sig"], rtol=0, atol=1e-10 * np.abs(g["cell_sig"]).max())
    np.testing.assert_allclose(vm, g["cell_vm"], rtol=0, atol=1e-10 * g["cell_vm"].max())
    np.testing.assert_allclose(nvm, g["nodal_vm"], rtol=0, atol=1e-10 * g["nodal_vm"].max())


def test_bsr3_pattern_is_3x3_expansion_of_reference_csr(golden):
    g = golden("tiny_block.npz")
    rp, ci, emap = solid.bsr3_pattern_and_map(g["conn"], len(g["nodes"]))
    R0 = _csr(g, "K0")
    assert 9 * len(ci) == R0.nnz
    B = sp.bsr_matrix((np.ones((len(ci), 3, 3)), ci, rp), shape=R0.shape).tocsr()
    B.sort_indices()
    assert (B.indptr == R0.indptr).all() and (B.indices == R0.indices).all()
    # every map entry hits the block (conn[e,a], conn[e,b])
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    conn = g["conn"]
    a_nodes = np.repeat(conn, 10, axis=1)
    b_nodes = np.tile(conn, (1, 10))
    assert (rows[emap] == a_nodes).all() and (ci[emap] == b_nodes).all()


def test_beam_oracle_matches_reference(golden):
    g = golden("beam_frame.npz")
    d = beam.batch_data(generate_frame_grid())
    f = beam.internal_forces(*d, g["U"])
    np.testing.assert_allclose(f, g["fint"], rtol=0, atol=1e-14 * np.abs(g["fint"]).max())


def test_reference_native_kernels_match_oracle(golden):
    """oracle/_ref (the reference's kernels.cpp compiled from source) vs the restatements."""
    import ctypes as C
    from pathlib import Path

    so = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libwnfea_ref_kernels.so"
    if not so.exists():
        pytest.skip("oracle/_ref not built (reference source absent)")
    lib = C.CDLL(str(so))
    g = golden("cantilever_c1.npz")
    nodes = np.ascontiguousarray(g["nodes"])
    conn = np.ascontiguousarray(g["conn"], dtype=np.int32)
    n = len(nodes)
    props = np.ascontiguousarray(np.tile([2.1e11, 0.3], (len(conn), 1)))
    U6 = np.random.default_rng(3).standard_normal(6 * n) * 1e-4
    F6 = np.zeros(6 * n)
    P = C.c_void_p
    lib.compute_c3d10_internal_forces_native.argtypes = [P, P, P, P, P, C.c_int, C.c_int]
    lib.compute_c3d10_internal_forces_native(nodes.ctypes.data, conn.ctypes.data, props.ctypes.data,
                                             U6.ctypes.data, F6.ctypes.data, len(conn), n)
    u3 = U6.reshape(n, 6)[:, :3].ravel()
    K0, _, _ = solid.assemble(nodes, conn, props, apply_bcs=False)
    f3 = K0 @ u3
    np.testing.assert_allclose(F6.reshape(n, 6)[:, :3].ravel(), f3, rtol=0, atol=1e-11 * np.abs(f3).max())
