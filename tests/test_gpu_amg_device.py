"""The AMG setup on the device (wn_amg_params.setup_on_device = 1, the default) against the host
builder (setup_on_device = 0, and the host-only wn_amg_setup_host).

Both builders share the aggregation and the per-aggregate QR (host code); the device builder
runs the diagonal, the power iterations, the smoothed prolongator, the transpose and the two
Galerkin products on the GPU with the host builder's summation order.  Checked per level: the
values of P, R and the coarse operators A_l against the host builder's (patterns equal up to
blocks whose terms cancel to an exact zero in one rounding and not the other), R = P^T
exactly, rho, 1/diag and the coarsest inverse; A_c against scipy's R (A P); and a solve with
each hierarchy (iteration counts within rounding noise).
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

from wnfea_b200.amg import AMGParams, export_system_hierarchy
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block
from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    a, b = sp.csr_matrix(a), sp.csr_matrix(b)
    return abs(a - b).max() <= tol * abs(b).max()


@pytest.mark.parametrize("which", ["c1", "ibeam"])
def test_device_setup_matches_host_builder(which):
    m = generate_c3d10_kuhn_block()[0] if which == "c1" else generate_c3d10_ibeam_structured(
        n_slices=24, length=4.0 * 24 / 315, seed=6)[0]
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    prm = AMGParams(coarse_size=300)
    s.amg_setup(AMGParams(**{**prm.__dict__, "setup_on_device": 0}))
    Hh = export_system_hierarchy(s)
    _, st_h = s.solve(F, rtol=1e-10, precision=0)
    s.amg_setup(AMGParams(**{**prm.__dict__, "setup_on_device": 1}))
    Hd = export_system_hierarchy(s)
    _, st_d = s.solve(F, rtol=1e-10, precision=0)
    assert len(Hd.levels) == len(Hh.levels) >= 1
    for lh, ld in zip(Hh.levels, Hd.levels):
        assert lh.bs == ld.bs and lh.n_nodes == ld.n_nodes
        assert abs(lh.rho - ld.rho) <= 1e-12 * lh.rho
        np.testing.assert_allclose(ld.dinv, lh.dinv, rtol=1e-13, atol=0)
        # Both builders drop all-zero blocks; a block whose terms cancel exactly can come out as
        # 0 in one summation order and as ~1e-17 in the other, so the patterns may differ by such
        # blocks: compare through the difference (a block present on one side only counts with
        # its full size) and bound the count of differing blocks.
        for a, b in ((ld.P, lh.P), (ld.R, lh.R)):
            assert _close(a, b, 1e-12)
            assert abs(a.nnz - b.nnz) <= 0.01 * b.nnz
        # R = P^T exactly (blocks transposed)
        assert abs(sp.csr_matrix(ld.R) - sp.csr_matrix(ld.P).T).max() == 0.0
        if lh.A is not None:
            assert _close(ld.A, lh.A, 1e-12)
            assert abs(ld.A.nnz - lh.A.nnz) <= 0.01 * lh.A.nnz
    # the Galerkin product of level 0 against scipy, and the coarsest inverse
    A0 = K.to_bsr().tocsr()
    P0, R0 = sp.csr_matrix(Hd.levels[0].P), sp.csr_matrix(Hd.levels[0].R)
    Ac = (R0 @ A0 @ P0).tocsr()
    A1 = sp.csr_matrix(Hd.levels[1].A) if len(Hd.levels) > 1 else sp.csr_matrix(Hd.coarse_A)
    assert _close(0.5 * (Ac + Ac.T), A1, 1e-12)
    np.testing.assert_allclose(Hd.coarse_inv, Hh.coarse_inv, rtol=0, atol=1e-9 * np.abs(Hh.coarse_inv).max())
    assert st_d["status"] == 0 and st_h["status"] == 0
    # hierarchies equal to ~1e-12 can move a tight-tolerance solve by an iteration or two
    assert abs(st_d["iterations"] - st_h["iterations"]) <= 2 + 0.05 * st_h["iterations"]


def test_device_setup_frame_system():
    """The 6-DOF fine level (beam frames): the device builder on row-major 6x6 blocks."""
    from wnfea_b200.beam import frame_linear_system
    from wnfea_b200.frames import generate_space_frame

    fm = generate_space_frame(8, 8, 8, seed=1)
    frame, system, F = frame_linear_system(fm)
    system.amg_setup(AMGParams(coarse_size=300, setup_on_device=0))
    uh, sth = system.solve(F, rtol=1e-10, precision="fp64")
    system.amg_setup(AMGParams(coarse_size=300, setup_on_device=1))
    ud, std = system.solve(F, rtol=1e-10, precision="fp64")
    assert sth["status"] == 0 and std["status"] == 0
    assert abs(std["iterations"] - sth["iterations"]) <= 2 + 0.05 * sth["iterations"]
    assert np.linalg.norm(ud - uh) <= 1e-8 * np.linalg.norm(uh)
    system.close()
    frame.close()
