"""GPU parity of the assembly, SpMV and element kernels against the oracle and the
reference's golden vectors (through the C ABI)."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import c3d10 as oc3d10
from oracle import solid
from wnfea_b200 import _lib
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block
from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector
from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, compute_c3d10_stress_field
from wnfea_b200.system import SolidSystem

pytestmark = pytest.mark.gpu


def _c1():
    m, _ = generate_c3d10_kuhn_block()
    return m


def test_element_stiffness_matches_reference(golden):
    g = golden("c3d10_element.npz")
    coords = np.ascontiguousarray(np.stack([g["tet"], g["curved"]]))
    props = np.array([[2.1e11, 0.3], [1.8e11, 0.33]])
    Ke = np.empty((2, 30, 30))
    _lib.call("wn_c3d10_element_stiffness", 2, _lib.ptr(coords), _lib.ptr(props), _lib.ptr(Ke))
    for k, ref in enumerate((g["Ke_tet"], g["Ke_curved"])):
        np.testing.assert_allclose(Ke[k], ref, rtol=0, atol=1e-14 * np.abs(ref).max())
        assert np.array_equal(Ke[k], Ke[k].T)  # exactly symmetric, as after c3d10.py:248


def test_assembly_no_bcs_matches_reference_csr(golden):
    g = golden("tiny_block.npz")
    s = SolidSystem(g["nodes"], g["conn"])
    s.assemble(np.tile([2.1e11, 0.3], (s.n_el, 1)), apply_bcs=False)
    rp, ci = s.pattern()
    K = sp.bsr_matrix((s.values(), ci, rp), shape=(3 * s.n_nodes,) * 2).tocsr()
    K.sort_indices()
    R = sp.csr_matrix((g["K0_data"], g["K0_indices"], g["K0_indptr"]), shape=K.shape)
    assert np.array_equal(K.indptr, R.indptr) and np.array_equal(K.indices, R.indices)
    np.testing.assert_allclose(K.data, R.data, rtol=0, atol=1e-14 * np.abs(R.data).max())


def test_assembly_with_bcs_matches_reference(golden):
    g = golden("cantilever_c1.npz")
    m = _c1()
    K, F, fixed = assemble_c3d10_sparse_3dof(m)
    assert list(fixed) == list(g["fixed"])
    np.testing.assert_array_equal(F, g["F"])
    Kc = K.tocsr()
    np.testing.assert_allclose(Kc @ g["v"], g["K_v"], rtol=0, atol=1e-13 * np.abs(g["K_v"]).max())
    np.testing.assert_allclose(Kc.diagonal(), g["K_diag"], rtol=1e-14)
    # full-matrix comparison against the oracle (same BC semantics)
    O, _, _ = solid.assemble(m.mesh_nodes, m.solid_elements, solid_element_props(m), solid_load_vector(m),
                             solid_fixed_dofs(m))
    D = (Kc - O).tocsr()
    assert np.abs(D.data).max(initial=0) <= 1e-14 * np.abs(O.data).max()


def test_pattern_and_map_match_oracle():
    m, _ = generate_c3d10_ibeam_structured(n_slices=8, length=4.0 * 8 / 315, seed=1)
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    rp, ci = s.pattern()
    orp, oci, oemap = solid.bsr3_pattern_and_map(m.solid_elements, len(m.mesh_nodes))
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    assert np.array_equal(s.element_map(), oemap)


def test_assembly_is_bit_reproducible():
    m, _ = generate_c3d10_ibeam_structured(n_slices=10, length=4.0 * 10 / 315, seed=2)
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    props = solid_element_props(m)
    s.assemble(props, apply_bcs=False)
    v1 = s.values().copy()
    s.assemble(props, apply_bcs=False)
    assert np.array_equal(v1, s.values())


@pytest.mark.parametrize("which", ["c1", "ibeam20"])
def test_assembled_matrix_is_exactly_symmetric(which):
    """K == K^T bit for bit, with and without the Dirichlet rows / columns: blocks (i, j) and
    (j, i) sum transposed terms in the same order, diagonal blocks are symmetric, and the split
    blocks (the vertex nodes' diagonal blocks, summed in chunks by several threads) are cut and
    combined alike; the graded modulus makes every element's lam, mu differ."""
    m = generate_c3d10_kuhn_block()[0] if which == "c1" else generate_c3d10_ibeam_structured(
        n_slices=20, length=4.0 * 20 / 315, seed=5)[0]
    props = solid_element_props(m)
    props[:, 0] *= np.exp(np.random.default_rng(1).uniform(-1, 1, len(props)))
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.set_fixed(solid_fixed_dofs(m))
    for bcs in (False, True):
        s.assemble(props, apply_bcs=bcs)
        rp, ci = s.pattern()
        K = solid.bsr3_to_csr(rp, ci, s.values())
        assert abs(K - K.T).max() == 0.0, bcs
        ovals = solid.bsr3_from_csr(solid.assemble(m.mesh_nodes, m.solid_elements, props, apply_bcs=False)[0], rp, ci)
        if not bcs:
            np.testing.assert_allclose(s.values(), ovals, rtol=0, atol=1e-14 * np.abs(ovals).max())


def test_jittered_ibeam_assembly_matches_oracle():
    m, _ = generate_c3d10_ibeam_structured(n_slices=12, length=4.0 * 12 / 315, seed=3)
    props = solid_element_props(m)
    props[:, 0] *= np.exp(np.random.default_rng(0).uniform(-1, 1, len(props)))  # graded modulus
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.assemble(props, apply_bcs=False)
    rp, ci = s.pattern()
    ovals = solid.bsr3_from_csr(solid.assemble(m.mesh_nodes, m.solid_elements, props, apply_bcs=False)[0], rp, ci)
    np.testing.assert_allclose(s.values(), ovals, rtol=0, atol=1e-14 * np.abs(ovals).max())


def test_spmv_fp64_fp32_match_scipy():
    import torch

    m, _ = generate_c3d10_ibeam_structured(n_slices=20, length=4.0 * 20 / 315, seed=4)
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    s.assemble(solid_element_props(m), apply_bcs=False)
    Kc = sp.bsr_matrix((s.values(), s.pattern()[1], s.pattern()[0]), shape=(3 * s.n_nodes,) * 2).tocsr()
    x = np.random.default_rng(5).standard_normal(3 * s.n_nodes)
    ref = Kc @ x
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    _lib.call("wn_spmv_solid_device", s.handle, 0, dx.data_ptr(), dy.data_ptr(), 0)
    torch.cuda.synchronize()
    np.testing.assert_allclose(dy.cpu().numpy(), ref, rtol=0, atol=1e-13 * np.abs(ref).max())
    dx32 = dx.float()
    dy32 = torch.empty_like(dx32)
    _lib.call("wn_spmv_solid_device", s.handle, 1, dx32.data_ptr(), dy32.data_ptr(), 0)
    torch.cuda.synchronize()
    err = np.abs(dy32.cpu().numpy().astype(np.float64) - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


@pytest.mark.parametrize("br,bc", [(3, 3), (6, 6), (3, 6), (6, 3)])
def test_generic_bsr_spmv_host_variant(br, bc):
    rng = np.random.default_rng(br * 10 + bc)
    n_rows, n_cols = 57, 41
    A = sp.random(n_rows, n_cols, density=0.15, random_state=1, format="csr")
    A.data[:] = 1.0
    A.sort_indices()
    rp = A.indptr.astype(np.int32)
    ci = A.indices.astype(np.int32)
    vals = rng.standard_normal((len(ci), br, bc))
    x = rng.standard_normal(n_cols * bc)
    y = rng.standard_normal(n_rows * br)
    B = sp.bsr_matrix((vals, ci, rp), shape=(n_rows * br, n_cols * bc))
    ref = 2.0 * (B @ x) + 0.5 * y
    _lib.call("wn_spmv_bsr_f64", br, bc, n_rows, n_cols, len(ci), _lib.ptr(rp), _lib.ptr(ci), _lib.ptr(vals),
              _lib.ptr(x), _lib.ptr(y), 2.0, 0.5)
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13)


def test_stress_field_matches_reference(golden):
    g = golden("cantilever_c1.npz")
    m = _c1()
    assemble_c3d10_sparse_3dof(m)
    sig, vm, nvm = compute_c3d10_stress_field(m, g["u_direct"])
    np.testing.assert_allclose(sig, g["cell_sig"], rtol=0, atol=1e-10 * np.abs(g["cell_sig"]).max())
    np.testing.assert_allclose(vm, g["cell_vm"], rtol=0, atol=1e-10 * g["cell_vm"].max())
    np.testing.assert_allclose(nvm, g["nodal_vm"], rtol=0, atol=1e-10 * g["nodal_vm"].max())


def test_internal_forces_reference_signature_stride6():
    """wn_c3d10_internal_forces keeps kernels.cpp's argument list and 6-DOF stride."""
    m = _c1()
    nodes = np.ascontiguousarray(m.mesh_nodes)
    conn = np.ascontiguousarray(m.solid_elements, dtype=np.int32)
    props = np.ascontiguousarray(solid_element_props(m))
    n = len(nodes)
    U6 = np.random.default_rng(3).standard_normal(6 * n) * 1e-4
    F6 = np.ones(6 * n)  # accumulated into, as the reference's += scatter
    _lib.call("wn_c3d10_internal_forces", _lib.ptr(nodes), _lib.ptr(conn), _lib.ptr(props), _lib.ptr(U6),
              _lib.ptr(F6), len(conn), n)
    K0, _, _ = solid.assemble(nodes, conn, props, apply_bcs=False)
    f3 = K0 @ U6.reshape(n, 6)[:, :3].ravel()
    got = F6.reshape(n, 6)
    np.testing.assert_allclose(got[:, :3].ravel() - 1.0, f3, rtol=0, atol=1e-12 * np.abs(f3).max())
    assert np.array_equal(got[:, 3:], np.ones((n, 3)))


def test_internal_forces_reference_signature_workspace_reuse():
    """The host-buffer call keeps its device buffers between calls: alternating meshes of
    different sizes give the device-resident kernel's bits every time; a bad node index is
    rejected."""
    meshes = [_c1(), generate_c3d10_ibeam_structured(n_slices=6, length=4.0 * 6 / 315, seed=2)[0]]
    ref = []
    for m in meshes:
        props = np.ascontiguousarray(solid_element_props(m))
        sysm = SolidSystem(m.mesh_nodes, m.solid_elements)
        sysm.assemble(props, apply_bcs=False)
        n = len(m.mesh_nodes)
        u = np.random.default_rng(n).standard_normal(3 * n) * 1e-4
        ref.append((m, props, u, sysm.internal_forces(u)))
    for m, props, u, f_dev in ref + ref[::-1]:
        n = len(m.mesh_nodes)
        U6 = np.zeros(6 * n)
        U6.reshape(n, 6)[:, :3] = u.reshape(n, 3)
        F6 = np.zeros(6 * n)
        _lib.call("wn_c3d10_internal_forces", _lib.ptr(np.ascontiguousarray(m.mesh_nodes)),
                  _lib.ptr(np.ascontiguousarray(m.solid_elements, dtype=np.int32)), _lib.ptr(props), _lib.ptr(U6),
                  _lib.ptr(F6), len(m.solid_elements), n)
        assert np.array_equal(F6.reshape(n, 6)[:, :3].ravel(), f_dev)
    m, props, u, _ = ref[0]
    bad = np.ascontiguousarray(m.solid_elements, dtype=np.int32).copy()
    bad[3, 4] = len(m.mesh_nodes)
    n = len(m.mesh_nodes)
    with pytest.raises(_lib.WnError):
        _lib.call("wn_c3d10_internal_forces", _lib.ptr(np.ascontiguousarray(m.mesh_nodes)), _lib.ptr(bad),
                  _lib.ptr(props), _lib.ptr(np.zeros(6 * n)), _lib.ptr(np.zeros(6 * n)), len(bad), n)


def test_internal_forces_and_adjoint_match_oracle():
    m, _ = generate_c3d10_ibeam_structured(n_slices=6, length=4.0 * 6 / 315, seed=8)
    props = solid_element_props(m)
    props[:, 0] *= np.exp(np.random.default_rng(1).uniform(-1, 1, len(props)))
    s = SolidSystem(m.mesh_nodes, m.solid_elements)
    fixed = solid_fixed_dofs(m)
    s.set_fixed(fixed)
    s.assemble(props, apply_bcs=True)
    u = np.random.default_rng(2).standard_normal(3 * s.n_nodes) * 1e-4
    f = s.internal_forces(u)
    K0, _, _ = solid.assemble(m.mesh_nodes, m.solid_elements, props, apply_bcs=False)
    np.testing.assert_allclose(f, K0 @ u, rtol=0, atol=1e-12 * np.abs(f).max())
    gE, gF = s.compliance_gradient(u)
    mask = np.zeros(3 * s.n_nodes, dtype=bool)
    mask[fixed] = True
    oE, oF = solid.compliance_gradient(m.mesh_nodes, m.solid_elements, props, u, mask)
    np.testing.assert_allclose(gE, oE, rtol=1e-12, atol=1e-12 * np.abs(oE).max())
    np.testing.assert_array_equal(gF, oF)


def test_inverted_element_is_rejected():
    m = _c1()
    conn = m.solid_elements.copy()
    conn[0, [1, 2]] = conn[0, [2, 1]]  # flip orientation of one element
    conn[0, [4, 5, 6, 7, 8, 9]] = conn[0, [6, 5, 4, 7, 9, 8]]
    s = SolidSystem(m.mesh_nodes, conn)
    with pytest.raises(_lib.WnError) as e:
        s.assemble(solid_element_props(m), apply_bcs=False)
    assert e.value.code == -3
