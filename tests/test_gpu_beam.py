"""GPU co-rotational beam path: internal force vs the reference's golden vector, consistent
tangent vs central differences of the oracle, linear stiffness at U = 0, Newton frame solve vs
the reference's 10-step JFNK solution."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import beam as obeam
from wnfea_b200 import _lib
from wnfea_b200.beam import BeamFrame, compute_internal_forces_fast, prepare_batch_data, solve_nonlinear_jfnk
from wnfea_b200.frames import generate_frame_grid

pytestmark = pytest.mark.gpu


def test_internal_force_matches_reference(golden):
    g = golden("beam_frame.npz")
    m = generate_frame_grid()
    f = compute_internal_forces_fast(m, g["U"])
    np.testing.assert_allclose(f, g["fint"], rtol=0, atol=1e-12 * np.abs(g["fint"]).max())
    # the reference's native signature, accumulating into F_int
    d = prepare_batch_data(m)
    F = np.ones(6 * d.n_nodes)
    _lib.call("wn_beam_internal_forces", _lib.ptr(d.nodes), _lib.ptr(d.beam_elements), _lib.ptr(d.beam_props),
              _lib.ptr(d.beam_e_ref), _lib.ptr(d.beam_L0), _lib.ptr(np.ascontiguousarray(g["U"])), _lib.ptr(F),
              d.n_beams, d.n_nodes)
    np.testing.assert_allclose(F - 1.0, g["fint"], rtol=0, atol=1e-11 * np.abs(g["fint"]).max())


@pytest.mark.parametrize("scale", [0.0, 1e-3, 5e-2])
def test_tangent_matches_central_differences(scale):
    """K_t = d f_int / dU (dual numbers) vs central differences of the oracle force (the check
    of test_nonlinear_jfnk.py:66-75), at U = 0 and at finite rotations."""
    m = generate_frame_grid(nx=4, ny=3)
    d = obeam.batch_data(m)
    n = 6 * len(m.mesh_nodes)
    U = np.random.default_rng(7).standard_normal(n) * scale
    fr = BeamFrame(m)
    fr.assemble_tangent(U, apply_bcs=False)
    Kt = fr.tangent_bsr().toarray()
    Kfd = obeam.tangent_fd(*d, U, h=1e-7)
    scale_k = np.abs(Kfd).max()
    assert np.abs(Kt - Kfd).max() <= 2e-6 * scale_k
    if scale == 0.0:  # the linearised frame is symmetric
        assert np.abs(Kt - Kt.T).max() <= 1e-9 * scale_k
    np.testing.assert_allclose(fr.internal_force(U), obeam.internal_forces(*d, U), rtol=0,
                               atol=1e-12 * max(1.0, np.abs(obeam.internal_forces(*d, U)).max()))


def test_bicgstab_solves_tangent_system():
    m = generate_frame_grid()
    fr = BeamFrame(m)
    n = fr.n
    mask = np.zeros(n, dtype=np.uint8)
    for s in m.supports:
        mask[6 * s.node_id : 6 * s.node_id + 6] = 1
    fr.set_fixed(mask)
    U = np.random.default_rng(1).standard_normal(n) * 1e-2
    U[mask.astype(bool)] = 0.0
    fr.assemble_tangent(U, apply_bcs=True)
    K = fr.tangent_bsr().tocsr()
    b = np.random.default_rng(2).standard_normal(n)
    x, its, rel, status = fr.solve(b, method="dense")
    assert status == 0
    assert np.linalg.norm(K @ x - b) <= 1e-9 * np.linalg.norm(b)
    np.testing.assert_allclose(x, np.linalg.solve(K.toarray(), b), rtol=0, atol=1e-8 * np.abs(x).max())
    # iterative path on a right-hand side in the range of the loads
    b2 = K @ (np.random.default_rng(3).standard_normal(n) * (1 - mask))
    x2, its2, rel2, status2 = fr.solve(b2, rtol=1e-8, max_iter=5000, method="bicgstab")
    assert status2 == 0 and np.linalg.norm(K @ x2 - b2) <= 2e-8 * np.linalg.norm(b2)


def test_newton_frame_matches_reference_jfnk(golden):
    g = golden("beam_frame.npz")
    m = generate_frame_grid()
    st = {}
    U = solve_nonlinear_jfnk(m, n_load_steps=10, tol_rel=1e-12, tol_abs=1e-8, verbose=False, stats=st)
    ref = g["U_nl"]
    # the reference stops at |R| < 1e-5 N (finite-difference JFNK); compare at that level
    assert np.abs(U - ref).max() <= 1e-5 * np.abs(ref).max()
    np.testing.assert_allclose(np.abs(U.reshape(-1, 6)[:, 2]).max(), 1.889e-2, rtol=2e-3)
    assert st["newton_iterations"] <= 40
