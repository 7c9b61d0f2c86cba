"""The library's host AMG setup (C++) checked on the CPU against scipy, and the oracle's
V-cycle/PCG with that hierarchy against the direct solution.  No GPU needed."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import spsolve

from oracle import amg as oamg
from oracle import solid
from wnfea_b200.amg import AMGParams, setup_host
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block
from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector


def _system(which):
    if which == "c1":
        m, _ = generate_c3d10_kuhn_block()
    elif which == "block":
        m, _ = generate_c3d10_kuhn_block(nx=12, ny=5, nz=7)
    else:
        m, _ = generate_c3d10_ibeam_structured(n_slices=12, length=4.0 * 12 / 315, seed=3)
    K, F, fixed = solid.assemble(m.mesh_nodes, m.solid_elements, solid_element_props(m), solid_load_vector(m),
                                 solid_fixed_dofs(m), apply_bcs=False)
    mask = np.zeros(K.shape[0], dtype=np.uint8)
    mask[fixed] = 1
    # BCs without eliminate_zeros: keep the 3x3 block pattern
    n = K.shape[0]
    row = np.repeat(np.arange(n), np.diff(K.indptr))
    mr, mc = mask[row].astype(bool), mask[K.indices].astype(bool)
    K.data[(mr | mc) & (row != K.indices)] = 0.0
    K.data[mr & (row == K.indices)] = 1.0
    F[mask.astype(bool)] = 0.0
    return m, K, F, mask


@pytest.fixture(scope="module", params=["c1", "ibeam"])
def case(request):
    m, K, F, mask = _system(request.param)
    H = setup_host(sp.bsr_matrix(K, blocksize=(3, 3)), m.mesh_nodes, mask, AMGParams(coarse_size=300))
    return m, K, F, mask, H


def test_hierarchy_is_galerkin(case):
    m, K, F, mask, H = case
    A = K
    assert len(H.levels) >= 1
    for lvl, L in enumerate(H.levels):
        P, R = L.P.tocsr(), L.R.tocsr()
        assert abs(R - P.T).max() == 0.0  # R = P^T exactly
        Ac = (R @ A @ P).toarray()
        nxt = H.levels[lvl + 1].A.toarray() if lvl + 1 < len(H.levels) else H.coarse_A
        scale = np.abs(Ac).max()
        np.testing.assert_allclose(nxt, 0.5 * (Ac + Ac.T), rtol=0, atol=1e-12 * scale)
        np.testing.assert_array_equal(nxt, nxt.T)
        d = A.diagonal()
        np.testing.assert_allclose(L.dinv, 1.0 / d, rtol=1e-15)
        A = sp.csr_matrix(nxt)


def test_spectral_radius_estimate(case):
    m, K, F, mask, H = case
    from scipy.sparse.linalg import eigsh

    d = K.diagonal()
    Ds = sp.diags(1 / np.sqrt(d))
    lam = eigsh(Ds @ K @ Ds, k=1, which="LA", return_eigenvectors=False)[0]
    rho = H.levels[0].rho
    assert 0.7 * lam <= rho <= lam * (1 + 1e-9)


def test_coarse_inverse(case):
    *_, H = case
    np.testing.assert_allclose(H.coarse_inv @ H.coarse_A, np.eye(len(H.coarse_A)), atol=1e-8)


def test_oracle_pcg_with_hierarchy_converges(case):
    m, K, F, mask, H = case
    u_ref = spsolve(K.tocsc(), F)
    x, its = oamg.pcg(K, F, lambda r: oamg.vcycle(K, H, r), rtol=1e-10, max_iter=300)
    assert its < 80, its
    assert np.linalg.norm(x - u_ref) / np.linalg.norm(u_ref) < 1e-8


def test_oracle_block_smoother_helpers_and_vcycle(case):
    """The oracle's block-Jacobi pieces behind the coarse-level change of basis: the block
    Cholesky (with its rule for a direction a block does not span), the block-diagonal inverse,
    and PCG with block smoothing on the 6-DOF levels reaching the direct solution."""
    m, K, F, mask, H = case
    rng = np.random.default_rng(4)
    M = rng.standard_normal((3, 6, 6))
    D = M @ np.transpose(M, (0, 2, 1)) + 6.0 * np.eye(6)
    D[1] = 0.0
    D[1, :3, :3] = 2.0 * np.eye(3)  # spans three of the six directions
    L = oamg.block_cholesky(D)
    for k in (0, 2):
        np.testing.assert_allclose(L[k] @ L[k].T, D[k], rtol=0, atol=1e-12 * np.abs(D[k]).max())
    np.testing.assert_allclose(L[1][:3, :3], np.sqrt(2.0) * np.eye(3))
    np.testing.assert_array_equal(L[1][3:, 3:], np.eye(3))
    A = sp.bsr_matrix((D, np.arange(3), np.arange(4)), shape=(18, 18)).tocsr()
    B = oamg.block_diag_inverse(A, 6).toarray()
    np.testing.assert_allclose(B[:6, :6] @ D[0], np.eye(6), atol=1e-12)
    if len(H.levels) < 2:
        return
    rhos = [None]
    for lv in range(1, len(H.levels)):
        Al = sp.csr_matrix(H.levels[lv].A)
        Li = np.linalg.inv(oamg.block_cholesky(oamg.diag_blocks(Al, 6)))
        n = Li.shape[0]
        T = sp.bsr_matrix((np.transpose(Li, (0, 2, 1)), np.arange(n), np.arange(n + 1)), shape=Al.shape)
        rhos.append(float(np.abs(np.linalg.eigvalsh((T.T @ Al @ T).toarray())).max()))
    u_ref = spsolve(K.tocsc(), F)
    x, its = oamg.pcg(K, F, lambda r: oamg.vcycle(K, H, r, block_rho=rhos), rtol=1e-10, max_iter=300)
    assert its < 80, its
    assert np.linalg.norm(x - u_ref) / np.linalg.norm(u_ref) < 1e-8


def test_setup_is_deterministic():
    m, K, F, mask = _system("c1")
    Kb = sp.bsr_matrix(K, blocksize=(3, 3))
    H1 = setup_host(Kb, m.mesh_nodes, mask, AMGParams(coarse_size=300))
    H2 = setup_host(Kb, m.mesh_nodes, mask, AMGParams(coarse_size=300))
    for a, b in zip(H1.levels, H2.levels):
        assert np.array_equal(a.P.data, b.P.data) and a.rho == b.rho
    assert np.array_equal(H1.coarse_inv, H2.coarse_inv)


_DUMP = r"""
import sys, numpy as np, scipy.sparse as sp
sys.path.insert(0, sys.argv[2])
from tests.test_amg_host import _system
from wnfea_b200.amg import AMGParams, setup_host
m, K, F, mask = _system("block")
H = setup_host(sp.bsr_matrix(K, blocksize=(3, 3)), m.mesh_nodes, mask, AMGParams(coarse_size=700))
out = {"coarse_A": H.coarse_A, "coarse_inv": H.coarse_inv}
for l, L in enumerate(H.levels):
    out[f"P{l}"] = L.P.data
    out[f"dinv{l}"] = L.dinv
    out[f"rho{l}"] = np.array([L.rho])
    if L.A is not None:
        out[f"A{l}"] = L.A.data
np.savez(sys.argv[1], **out)
"""


def test_setup_is_identical_for_any_thread_count(tmp_path):
    """The host setup (aggregation, smoothed prolongator, Galerkin products, dense coarsest
    Cholesky and inverse) in two processes with 1 and 5 host threads: every exported array is
    bit-identical.  The mesh is large enough (4,125 nodes, coarsest > 64 DOFs) for the row and
    interleaved parallel loops to split."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    res = []
    for nth in ("1", "5"):
        f = tmp_path / f"h{nth}.npz"
        env = dict(os.environ, WN_HOST_THREADS=nth)
        subprocess.run([sys.executable, "-c", _DUMP, str(f), str(root)], check=True, env=env, cwd=root, timeout=600)
        res.append(np.load(f))
    a, b = res
    assert sorted(a.files) == sorted(b.files) and a["coarse_inv"].shape[0] > 64
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
