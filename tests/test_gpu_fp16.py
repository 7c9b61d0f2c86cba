"""The FP16 V-cycle (solve precision 3, "mixed_fp16", the reference's TRI_PRECISION preconditioner,
wnfea/solver/mixed_precision.py:96-103): the fine level smooths with the equilibrated matrix
S K S (S = diag(K)^-1/2) stored in FP16.  Checked against the oracle V-cycle run on the same
FP16-rounded matrix, against scipy's direct solve, and for its refresh after a re-assembly."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import spsolve

from oracle import amg as oamg
from oracle import solid
from wnfea_b200 import TRI_PRECISION, _lib
from wnfea_b200.amg import AMGParams, export_system_hierarchy
from wnfea_b200.mesh import generate_c3d10_ibeam_structured, generate_c3d10_kuhn_block
from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector
from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_pcg, solve_c3d10_system

pytestmark = pytest.mark.gpu


def _ibeam(n_slices=16, seed=3):
    m, _ = generate_c3d10_ibeam_structured(n_slices=n_slices, length=4.0 * n_slices / 315, seed=seed)
    return m


def _fp16_level0(K):
    """S^-1 fp16(S K S) S^-1: the fine matrix the FP16 V-cycle smooths with, in the original
    scaling (S K S formed in FP64 and rounded to FP16 once, as the library's pack)."""
    K = K.tocsr()
    s = 1.0 / np.sqrt(K.diagonal())
    Kh = (sp.diags(s) @ K @ sp.diags(s)).tocsr()
    Kh.data = Kh.data.astype(np.float16).astype(np.float64)
    return (sp.diags(1.0 / s) @ Kh @ sp.diags(1.0 / s)).tocsr()


@pytest.mark.parametrize("which", ["c1", "ibeam"])
@pytest.mark.parametrize("degree", [1, 2])
def test_fp16_vcycle_matches_oracle(which, degree):
    import torch

    m = generate_c3d10_kuhn_block()[0] if which == "c1" else _ibeam()
    K, F, fixed = assemble_c3d10_sparse_3dof(m)
    s = K.system
    prm = AMGParams(coarse_size=300, smoother_degree=degree, cheb_lower=1.0 / 16.0 if degree == 1 else 1.0 / 30.0)
    s.amg_setup(prm)
    H = export_system_hierarchy(s)
    Kfull = K.to_bsr().tocsr()
    K16 = _fp16_level0(Kfull)
    assert abs(K16 - Kfull).max() > 0  # the FP16 rounding is not a no-op
    r = np.random.default_rng(1).standard_normal(K.shape[0])
    z_ref = oamg.vcycle(K16, H, r, degree=degree, dtype=np.float32, lower=prm.cheb_lower, safety=prm.cheb_safety)
    dr = torch.from_numpy(r).cuda().float()
    dz = torch.empty_like(dr)
    _lib.call("wn_amg_vcycle_device", s.handle, 3, dr.data_ptr(), dz.data_ptr(), 0)
    torch.cuda.synchronize()
    z = dz.cpu().numpy().astype(np.float64)
    err = np.linalg.norm(z - z_ref) / np.linalg.norm(z_ref)
    assert err < 1e-4, err
    assert r @ z > 0


def test_fp16_solve_matches_direct_and_fp32_iterations():
    m = _ibeam(24, seed=7)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    Ko, Fo = solid.assemble(m.mesh_nodes, m.solid_elements, solid_element_props(m), solid_load_vector(m),
                            solid_fixed_dofs(m))[:2]
    u_ref = spsolve(Ko.tocsc(), Fo)
    u16, st16 = solve_c3d10_system(K, F, method="pcg", rtol=1e-8, preconditioner="amg", precision="mixed_fp16")
    u32, st32 = solve_c3d10_system(K, F, method="pcg", rtol=1e-8, preconditioner="amg", precision="mixed_fp32")
    assert st16["status"] == 0 and st16["rel_res"] < 1e-8
    assert np.linalg.norm(Fo - Ko @ u16) <= 1e-8 * np.linalg.norm(Fo) * 1.01  # host true residual
    assert np.linalg.norm(u16 - u_ref) / np.linalg.norm(u_ref) < 1e-6
    assert st16["iterations"] <= 1.15 * st32["iterations"] + 2, (st16["iterations"], st32["iterations"])
    # deterministic
    u16b, _ = solve_c3d10_system(K, F, method="pcg", rtol=1e-8, preconditioner="amg", precision="mixed_fp16")
    assert np.array_equal(u16, u16b)


def test_fp16_pack_follows_reassembly():
    """A re-assembly with other material values rebuilds the FP16 pack before the next solve."""
    m = _ibeam(12, seed=5)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    s.amg_setup()
    u_a, st_a = s.solve(F, rtol=1e-9, precision=3)
    props = s.props.copy()
    props[::2, 0] *= 3.0
    s.assemble(props)  # the hierarchy stays; the fine level follows the new values
    u_b, st_b = s.solve(F, rtol=1e-9, precision=3)
    u_c, st_c = s.solve(F, rtol=1e-9, precision=0)
    assert st_a["status"] == st_b["status"] == st_c["status"] == 0
    assert np.linalg.norm(u_b - u_c) <= 1e-7 * np.linalg.norm(u_c)
    assert np.linalg.norm(u_b - u_a) > 1e-3 * np.linalg.norm(u_a)


def test_fp16_mode_arguments():
    m = _ibeam(8, seed=2)
    K, F, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    s.amg_setup()
    with pytest.raises(ValueError):
        solve_c3d10_pcg(K, F, rtol=1e-8, preconditioner="jacobi", precision="mixed_fp16")
    with pytest.raises(_lib.WnError):  # WN_EINVAL from the library: FP16 V-cycle without AMG
        s.solve(F, rtol=1e-8, precond=1, precision=3)
    s.set_streaming(False)  # the FP16 fine level exists only streamed
    with pytest.raises(_lib.WnError):
        s.solve(F, rtol=1e-8, precision=3)
    s.set_streaming(True)
    u, st = s.solve(F, rtol=1e-8, precision=3)
    assert st["status"] == 0
    assert TRI_PRECISION.solver_precision == "mixed_fp16"
