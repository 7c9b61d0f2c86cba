"""Element-level C3D10 API (element_stiffness/internal_forces/stresses_c3d10, the reference's
wnfea/elements/c3d10.py:219-318) on the GPU against the reference's golden outputs and the
oracle."""

from __future__ import annotations

import numpy as np
import pytest

import wnfea_b200 as wn
from oracle import c3d10 as oc3d10

pytestmark = pytest.mark.gpu


def _tol(ref):
    return 1e-13 * max(np.abs(ref).max(), 1e-300)


def test_single_element_matches_reference(golden):
    g = golden("c3d10_element.npz")
    Ke = wn.element_stiffness_c3d10(g["curved"], 1.8e11, 0.33)
    assert Ke.shape == (30, 30)
    np.testing.assert_allclose(Ke, g["Ke_curved"], rtol=0, atol=_tol(g["Ke_curved"]))
    assert np.array_equal(Ke, Ke.T)
    f = wn.element_internal_forces_c3d10(g["curved"], g["u_e"], 1.8e11, 0.33)
    assert f.shape == (30,)
    np.testing.assert_allclose(f, g["fint_curved"], rtol=0, atol=_tol(g["fint_curved"]))
    sig, vm, vmax = wn.element_stresses_c3d10(g["curved"], g["u_e"], 2.0e11, 0.28)
    assert sig.shape == (4, 6) and vm.shape == (4,) and isinstance(vmax, float)
    np.testing.assert_allclose(sig, g["sig_gp"], rtol=0, atol=_tol(g["sig_gp"]))
    np.testing.assert_allclose(vm, g["vm_gp"], rtol=0, atol=_tol(g["vm_gp"]))
    assert vmax == float(np.max(vm))


def test_element_batch_matches_oracle(golden):
    g = golden("c3d10_element.npz")
    rng = np.random.default_rng(7)
    m = 257
    base = np.where(rng.random(m)[:, None, None] < 0.5, g["tet"], g["curved"])
    coords = base * rng.uniform(0.5, 2.0, (m, 1, 1)) + rng.standard_normal((m, 1, 3))
    u = rng.standard_normal((m, 30)) * 1e-3
    E = rng.uniform(1e9, 3e11, m)
    nu = rng.uniform(0.0, 0.45, m)
    props = np.stack([E, nu], axis=1)
    Ke = wn.element_stiffness_c3d10(coords, E, nu)
    f = wn.element_internal_forces_c3d10(coords, u, E, nu)
    sig, vm, vmax = wn.element_stresses_c3d10(coords, u, E, nu)
    Ke_o = oc3d10.element_stiffness_batch(coords, props)
    f_o = oc3d10.element_internal_forces_batch(coords, u, props)
    sig_o, vm_o = oc3d10.element_stresses_batch(coords, u, props)[:2]
    assert Ke.shape == (m, 30, 30) and f.shape == (m, 30) and sig.shape == (m, 4, 6) and vmax.shape == (m,)
    for e in range(m):
        np.testing.assert_allclose(Ke[e], Ke_o[e], rtol=0, atol=_tol(Ke_o[e]))
        np.testing.assert_allclose(f[e], f_o[e], rtol=0, atol=1e-12 * np.abs(f_o[e]).max())
        np.testing.assert_allclose(sig[e], sig_o[e], rtol=0, atol=1e-12 * np.abs(sig_o[e]).max())
        np.testing.assert_allclose(vm[e], vm_o[e], rtol=1e-12)
    assert np.array_equal(vmax, vm.max(axis=1))
    # scalar material broadcast over the batch equals the per-element arrays
    assert np.array_equal(wn.element_stiffness_c3d10(coords[:5], 2e11, 0.3),
                          wn.element_stiffness_c3d10(coords[:5], np.full(5, 2e11), np.full(5, 0.3)))
