"""Block-Jacobi smoothing of the AMG's 6-DOF levels (wn_amg_params.coarse_block_smoother = 1,
the default) against the point-basis hierarchy of the same setup (coarse_block_smoother = 0).

The GPU setup moves every level below the finest to the basis in which its 6 x 6 diagonal
blocks are the identity: with D_i = L_i L_i^T the diagonal block of node i of A_l and
T_l = diag(L_i^-T),  A^_l = T_l^T A_l T_l,  P^_l = T_l^-1 P_l T_(l+1),  R^_l = P^_l^T  (T_0 and
the dense coarsest level's T are the identity).  The point smoother on A^_l is then the block
smoother on A_l.  Checked on the host: the operators against T from the oracle's block
Cholesky of the point-basis levels, R^ = P^^T and A^ = A^^T exactly, identity diagonal blocks; the V-cycle against the
oracle's block-Jacobi V-cycle on the point-basis levels; and the solve.
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import amg as oamg
from wnfea_b200 import _lib
from wnfea_b200.amg import AMGParams, export_system_hierarchy
from wnfea_b200.mesh import generate_c3d10_ibeam_structured
from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof

pytestmark = pytest.mark.gpu


def _basis(A, bs):
    """T = diag(L_i^-T) and T^-1 = diag(L_i^T) from the diagonal blocks of A."""
    L = oamg.block_cholesky(oamg.diag_blocks(A, bs))
    Linv = np.linalg.inv(L)
    n = L.shape[0]
    T = sp.bsr_matrix((np.transpose(Linv, (0, 2, 1)), np.arange(n), np.arange(n + 1)), shape=A.shape).tocsr()
    Ti = sp.bsr_matrix((np.transpose(L, (0, 2, 1)), np.arange(n), np.arange(n + 1)), shape=A.shape).tocsr()
    return T, Ti


def _rel(a, b):
    a, b = sp.csr_matrix(a), sp.csr_matrix(b)
    return abs(a - b).max() / abs(b).max()


def test_coarse_block_basis_operators_vcycle_and_solve():
    import torch

    m, _ = generate_c3d10_ibeam_structured(n_slices=16, length=4.0 * 16 / 315, seed=3)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    prm = AMGParams(coarse_size=300)
    s.amg_setup(AMGParams(**{**prm.__dict__, "coarse_block_smoother": 0}))
    Hp = export_system_hierarchy(s)
    u_p, st_p = s.solve(F, rtol=1e-10, precision=0)
    s.amg_setup(prm)
    Hb = export_system_hierarchy(s)
    u_b, st_b = s.solve(F, rtol=1e-10, precision=0)
    nlev = len(Hp.levels)
    assert nlev == len(Hb.levels) >= 2

    # the basis of each 6-DOF level from the point-basis matrices
    T = [None] + [_basis(Hp.levels[lv].A, 6) for lv in range(1, nlev)] + [None]
    assert Hb.levels[0].rho == Hp.levels[0].rho
    np.testing.assert_array_equal(Hb.levels[0].dinv, Hp.levels[0].dinv)
    for lv in range(nlev):
        Pp, Pb, Rb = (sp.csr_matrix(x) for x in (Hp.levels[lv].P, Hb.levels[lv].P, Hb.levels[lv].R))
        left = T[lv][1] if T[lv] is not None else sp.identity(Pp.shape[0], format="csr")
        right = T[lv + 1][0] if T[lv + 1] is not None else sp.identity(Pp.shape[1], format="csr")
        assert _rel(Pb, left @ Pp @ right) <= 1e-12
        assert abs(Rb - Pb.T).max() == 0.0  # R^ = P^^T bitwise
        if lv == 0:
            continue
        Ab = sp.csr_matrix(Hb.levels[lv].A)
        Ap = sp.csr_matrix(Hp.levels[lv].A)
        Tl = T[lv][0]
        assert _rel(Ab, Tl.T @ Ap @ Tl) <= 1e-12
        assert abs(Ab - Ab.T).max() == 0.0  # exactly symmetric
        # identity diagonal blocks: 1 / diag = 1 up to rounding
        np.testing.assert_allclose(Hb.levels[lv].dinv, 1.0, rtol=0, atol=1e-12)
        # rho of the new basis = rho(D_block^-1 A_l), estimated by power iterations from below
        if Ab.shape[0] <= 4000:
            lam = np.linalg.eigvalsh((Tl.T @ Ap @ Tl).toarray()).max()
            assert 0.7 * lam <= Hb.levels[lv].rho <= (1 + 1e-9) * lam

    # V-cycle: the GPU's on the new basis = the oracle's block-Jacobi V-cycle on the old basis.
    # The output of one V-cycle is dominated by the coarsest solve's low modes, so the smoother of
    # the 6-DOF levels shows in the energy norm |v|_K = sqrt(v^T K v) (point against block: about
    # 1e-5 of |z|_K on this beam); the GPU must match the oracle far below that.
    Kfull = K.to_bsr().tocsr()

    def en(v):
        return np.sqrt(abs(v @ (Kfull @ v)))

    r = np.random.default_rng(1).standard_normal(K.shape[0])
    rhos = [None] + [Hb.levels[lv].rho for lv in range(1, nlev)]
    z_ref = oamg.vcycle(Kfull, Hp, r, degree=1, lower=prm.cheb_lower, safety=prm.cheb_safety, block_rho=rhos)
    z_pt = oamg.vcycle(Kfull, Hp, r, degree=1, lower=prm.cheb_lower, safety=prm.cheb_safety)
    gap = en(z_pt - z_ref) / en(z_ref)
    assert gap > 1e-7
    dr = torch.from_numpy(r).cuda()
    dz = torch.empty_like(dr)
    _lib.call("wn_amg_vcycle_device", s.handle, 0, dr.data_ptr(), dz.data_ptr(), 0)
    torch.cuda.synchronize()
    z = dz.cpu().numpy()
    assert np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref) < 1e-10
    assert en(z - z_ref) / en(z_ref) < 1e-4 * gap
    dr32 = dr.float()
    dz32 = torch.empty_like(dr32)
    _lib.call("wn_amg_vcycle_device", s.handle, 1, dr32.data_ptr(), dz32.data_ptr(), 0)
    torch.cuda.synchronize()
    z32 = dz32.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(z32 - z_ref) / np.linalg.norm(z_ref) < 1e-4
    assert en(z32 - z_ref) / en(z_ref) < 0.1 * gap

    # both solves converge to the same solution; the block smoother needs no more iterations
    assert st_p["status"] == 0 and st_b["status"] == 0
    assert st_b["iterations"] <= st_p["iterations"] + 1
    assert np.linalg.norm(u_b - u_p) <= 1e-8 * np.linalg.norm(u_p)
