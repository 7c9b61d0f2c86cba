"""Compliance adjoint through torch.autograd on the GPU, checked against central finite
differences of the GPU solve and against the oracle's FP64 gradient."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.sparse.linalg import spsolve

from oracle import solid
from wnfea_b200.autograd import ComplianceProblem
from wnfea_b200.mesh import generate_c3d10_pressure_block
from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def block():
    import torch

    m, _ = generate_c3d10_pressure_block(nx=8, ny=4, nz=3, seed=3)  # 576 elements
    props = solid_element_props(m)
    prob = ComplianceProblem.from_model(m, precision="fp64", rtol=1e-11)
    E = torch.from_numpy(props[:, 0].copy()).cuda().requires_grad_(True)
    F = torch.from_numpy(solid_load_vector(m)).cuda().requires_grad_(True)
    return m, props, prob, E, F


def test_autograd_matches_oracle_gradient(block):
    import torch

    m, props, prob, E, F = block
    C = prob.compliance(E, F)
    C.backward()
    K, Fo, fixed = solid.assemble(m.mesh_nodes, m.solid_elements, props, solid_load_vector(m), solid_fixed_dofs(m))
    u = spsolve(K.tocsc(), Fo)
    mask = np.zeros(len(Fo), dtype=bool)
    mask[fixed] = True
    gE_ref, gF_ref = solid.compliance_gradient(m.mesh_nodes, m.solid_elements, props, u, mask)
    np.testing.assert_allclose(float(C.detach()), Fo @ u, rtol=1e-9)
    gE = E.grad.cpu().numpy()
    gF = F.grad.cpu().numpy()
    assert np.abs(gE - gE_ref).max() <= 1e-8 * np.abs(gE_ref).max()
    assert np.abs(gF - gF_ref).max() <= 1e-8 * np.abs(gF_ref).max()
    assert (gE < 0).all()  # stiffening any element lowers the compliance
    E.grad = None
    F.grad = None


def test_gradient_matches_central_differences(block):
    """Central differences of the energy-consistent compliance 2F.u - u.Ku (error quadratic
    in the solve error) on 8 seeded elements, h = 1e-3 E_e."""
    import torch

    m, props, prob, E, F = block
    E0 = E.detach().clone()
    u, Fb = prob.solve(E0, F.detach())
    gE, gF = prob.gradient(u)
    gE = gE.cpu().numpy()
    rng = np.random.default_rng(0)
    for e in rng.choice(len(E0), size=8, replace=False):
        h = 1e-3 * float(E0[e])
        vals = []
        for sgn in (1.0, -1.0):
            Ep = E0.clone()
            Ep[e] += sgn * h
            up, Fbp = prob.solve(Ep, F.detach())
            vals.append(prob.energy_compliance(up, Fbp))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - gE[e]) <= 1e-5 * abs(gE[e]), (e, fd, gE[e])
    # load direction: dC/dF . d = 2 u . d
    d = torch.randn_like(F.detach())
    eps = 1e-3 * float(F.detach().abs().max())
    cp = prob.energy_compliance(*prob.solve(E0, F.detach() + eps * d))
    cm = prob.energy_compliance(*prob.solve(E0, F.detach() - eps * d))
    fd = (cp - cm) / (2 * eps)
    an = float(torch.dot(gF, d))
    assert abs(fd - an) <= 1e-6 * abs(an)


def test_mixed_precision_forward_and_hierarchy_reuse(block):
    import torch

    m, props, _, E, F = block
    prob = ComplianceProblem.from_model(m, precision="mixed_fp32", rtol=1e-8, reuse_hierarchy=True)
    c1 = float(prob.compliance(E.detach(), F.detach()))
    E2 = E.detach() * 1.5  # stiffer everywhere: C scales by 1/1.5, same hierarchy reused
    c2 = float(prob.compliance(E2, F.detach()))
    assert prob.last_stats["status"] == 0
    np.testing.assert_allclose(c2, c1 / 1.5, rtol=1e-7)
