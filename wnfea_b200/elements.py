"""Element-level C3D10 operators on the GPU (the reference's wnfea/elements/c3d10.py:219-318).

``element_stiffness_c3d10``, ``element_internal_forces_c3d10`` and ``element_stresses_c3d10``
keep the reference's names, arguments and return types for one element ((10, 3) coordinates,
scalar E and nu).  Each also takes a batch -- coordinates (M, 10, 3), displacements (M, 30),
E and nu scalars or (M,) arrays -- and then returns the stacked results, so that many elements
go to the device in one call.  Every call runs the library's kernels (the Gauss-point
derivatives, the FP64 products and the von Mises reduction of the mesh-level operators);
the inputs and outputs are host arrays.
"""

from __future__ import annotations

import numpy as np

from ._lib import call, ptr


def _coords(node_coords) -> tuple[np.ndarray, bool]:
    c = np.ascontiguousarray(node_coords, dtype=np.float64)
    if c.shape == (10, 3):
        return c[None], True
    if c.ndim == 3 and c.shape[1:] == (10, 3):
        return c, False
    raise ValueError(f"Expected node_coords of shape (10, 3) or (M, 10, 3), got {c.shape}")


def _props(E, nu, m: int) -> np.ndarray:
    props = np.empty((m, 2), dtype=np.float64)
    props[:, 0] = np.broadcast_to(np.asarray(E, dtype=np.float64), (m,))
    props[:, 1] = np.broadcast_to(np.asarray(nu, dtype=np.float64), (m,))
    return props


def _disp(u_e, m: int) -> np.ndarray:
    u = np.ascontiguousarray(u_e, dtype=np.float64)
    if u.size != 30 * m:
        raise ValueError(f"Expected u_e with {30 * m} entries ((30,) per element), got shape {u.shape}")
    return u.reshape(m, 30)


def element_stiffness_c3d10(node_coords, E, nu) -> np.ndarray:
    """30x30 element stiffness K_e = sum_g w_g B_g^T C B_g det J_g (c3d10.py:219-249), exactly
    symmetric; (M, 30, 30) for a batch."""
    c, single = _coords(node_coords)
    m = len(c)
    Ke = np.empty((m, 30, 30), dtype=np.float64)
    call("wn_c3d10_element_stiffness", m, ptr(c), ptr(_props(E, nu, m)), ptr(Ke))
    return Ke[0] if single else Ke


def element_internal_forces_c3d10(node_coords, u_e, E, nu) -> np.ndarray:
    """f_int = sum_g w_g B_g^T C B_g u_e det J_g (c3d10.py:252-283); (M, 30) for a batch."""
    c, single = _coords(node_coords)
    m = len(c)
    u = _disp(u_e, m)
    # every element on its own ten nodes: node 10 e + a, DOF stride 6 (the mesh-level entry's)
    nodes = c.reshape(m * 10, 3)
    conn = np.arange(m * 10, dtype=np.int32).reshape(m, 10)
    U = np.zeros((m * 10, 6), dtype=np.float64)
    U[:, :3] = u.reshape(m * 10, 3)
    F = np.zeros_like(U)
    call("wn_c3d10_internal_forces", ptr(nodes), ptr(conn), ptr(_props(E, nu, m)), ptr(U), ptr(F), m, m * 10)
    f = np.ascontiguousarray(F[:, :3]).reshape(m, 30)
    return f[0] if single else f


def element_stresses_c3d10(node_coords, u_e, E, nu):
    """Gauss-point Cauchy stresses (4, 6) [sxx, syy, szz, sxy, syz, szx], von Mises (4,) and
    their maximum (c3d10.py:286-318); for a batch (M, 4, 6), (M, 4) and (M,)."""
    c, single = _coords(node_coords)
    m = len(c)
    u = _disp(u_e, m)
    sig = np.empty((m, 4, 6), dtype=np.float64)
    vm = np.empty((m, 4), dtype=np.float64)
    call("wn_c3d10_element_stresses", m, ptr(c), ptr(_props(E, nu, m)), ptr(u), ptr(sig), ptr(vm))
    if single:
        return sig[0], vm[0], float(np.max(vm[0]))
    return sig, vm, vm.max(axis=1)
