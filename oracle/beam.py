"""ORACLE (test infrastructure only) -- FP64 CPU restatement of the co-rotational beam path.

Nothing in the product imports this module.

* ``batch_data``      -- reference triads, lengths and section/material rows as
                         prepare_batch_data builds them (wnfea/solver/fast_kernels.py:263-306):
                         e2 = ref x e1 with ref = z unless |e1_z| >= 0.9 (then y), e3 = e1 x e2;
                         props [E, G, A, Iy, Iz, J];
* ``internal_forces`` -- the vectorised co-rotational internal force of
                         compute_internal_forces_fast's NumPy branch (fast_kernels.py:451-537):
                         Rodrigues rotation of the reference triad onto the current chord,
                         average twist, Gram-Schmidt, local [N, My1, Mz1, Tx, My2, Mz2] and
                         f = B^T q scattered at 6 DOF / node;
* ``linear_stiffness``-- assembled T^T K_l T of the linear 12x12 beam
                         (wnfea/solver/assembler.py:13-148), the tangent at U = 0.
"""

from __future__ import annotations

import numpy as np


def batch_data(model):
    nodes = np.asarray(model.mesh_nodes, dtype=np.float64)
    el = np.asarray(model.mesh_elements, dtype=np.int64)
    props = np.zeros((len(el), 6))
    for e in range(len(el)):
        a = model.element_properties[e]
        m = model.materials[a.material_name]
        s = model.sections[a.section_name]
        props[e] = [m.youngs_modulus, m.shear_modulus, s.area, s.iy, s.iz, s.j]
    v0 = nodes[el[:, 1]] - nodes[el[:, 0]]
    L0 = np.linalg.norm(v0, axis=1)
    e1 = v0 / np.maximum(L0[:, None], 1e-15)
    eref = np.zeros((len(el), 9))
    for i in range(len(el)):
        ref = np.array([0.0, 0.0, 1.0]) if abs(e1[i, 2]) < 0.9 else np.array([0.0, 1.0, 0.0])
        e2 = np.cross(ref, e1[i])
        e2 /= np.linalg.norm(e2)
        e3 = np.cross(e1[i], e2)
        e3 /= np.linalg.norm(e3)
        eref[i] = np.concatenate([e1[i], e2, e3])
    return nodes, el, props, eref, L0


def internal_forces(nodes, el, props, eref, L0, U):
    n1, n2 = el[:, 0], el[:, 1]
    v0 = nodes[n2] - nodes[n1]
    e1_0, e2_0, e3_0 = eref[:, 0:3], eref[:, 3:6], eref[:, 6:9]
    Un = U.reshape(-1, 6)
    u1, th1, u2, th2 = Un[n1, :3], Un[n1, 3:], Un[n2, :3], Un[n2, 3:]
    du = u2 - u1
    v = v0 + du
    L = np.linalg.norm(v, axis=1)
    r1 = v / np.maximum(L[:, None], 1e-15)
    cr = np.cross(e1_0, r1)
    sphi = np.linalg.norm(cr, axis=1)
    cphi = np.sum(e1_0 * r1, axis=1)
    r2, r3 = e2_0.copy(), e3_0.copy()
    m = sphi > 1e-12
    if np.any(m):
        ax = cr[m] / sphi[m, None]
        phi = np.arctan2(sphi[m], cphi[m])
        cp, sp_ = np.cos(phi)[:, None], np.sin(phi)[:, None]
        r2[m] = e2_0[m] * cp + np.cross(ax, e2_0[m]) * sp_ + ax * np.sum(ax * e2_0[m], 1, keepdims=True) * (1 - cp)
        r3[m] = e3_0[m] * cp + np.cross(ax, e3_0[m]) * sp_ + ax * np.sum(ax * e3_0[m], 1, keepdims=True) * (1 - cp)
    tw = 0.5 * np.sum((th1 + th2) * r1, axis=1)
    ct, st = np.cos(tw)[:, None], np.sin(tw)[:, None]
    r2, r3 = r2 * ct + np.cross(r1, r2) * st, r3 * ct + np.cross(r1, r3) * st
    r1 = r1 / np.linalg.norm(r1, axis=1, keepdims=True)
    r2 = r2 - np.sum(r2 * r1, axis=1, keepdims=True) * r1
    r2 = r2 / np.linalg.norm(r2, axis=1, keepdims=True)
    r3 = np.cross(r1, r2)
    r3 = r3 / np.linalg.norm(r3, axis=1, keepdims=True)
    ul = (2.0 * np.sum(v0 * du, 1) + np.sum(du * du, 1)) / (L + L0)
    thy1 = np.sum(r2 * th1, 1) + np.sum(r3 * du, 1) / L
    thz1 = np.sum(r3 * th1, 1) - np.sum(r2 * du, 1) / L
    thx = np.sum(r1 * (th2 - th1), 1)
    thy2 = np.sum(r2 * th2, 1) + np.sum(r3 * du, 1) / L
    thz2 = np.sum(r3 * th2, 1) - np.sum(r2 * du, 1) / L
    E, G, A, Iy, Iz, J = props.T
    N = E * A / L0 * ul
    My1 = E * Iy / L0 * (4 * thy1 + 2 * thy2)
    My2 = E * Iy / L0 * (2 * thy1 + 4 * thy2)
    Mz1 = E * Iz / L0 * (4 * thz1 + 2 * thz2)
    Mz2 = E * Iz / L0 * (2 * thz1 + 4 * thz2)
    Tx = G * J / L0 * thx
    f1 = -N[:, None] * r1 - ((My1 + My2) / L)[:, None] * r3 + ((Mz1 + Mz2) / L)[:, None] * r2
    m1 = -Tx[:, None] * r1 + My1[:, None] * r2 + Mz1[:, None] * r3
    m2 = Tx[:, None] * r1 + My2[:, None] * r2 + Mz2[:, None] * r3
    F = np.zeros((len(nodes), 6))
    np.add.at(F, n1, np.hstack([f1, m1]))
    np.add.at(F, n2, np.hstack([-f1, m2]))
    return F.ravel()


def tangent_fd(nodes, el, props, eref, L0, U, h=1e-7):
    """Central-difference tangent dF_int/dU (dense), the check used by
    test_nonlinear_jfnk.py:66-75 for the JFNK operator."""
    n = U.size
    K = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = h
        K[:, j] = (internal_forces(nodes, el, props, eref, L0, U + e) - internal_forces(nodes, el, props, eref, L0, U - e)) / (2 * h)
    return K
