"""ORACLE (test infrastructure only) -- FP64 CPU restatement of the reference's C3D10 element.

Nothing in the product imports this module.  Tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it as the checker.

Follows wnfea/elements/c3d10.py, vectorised over elements with NumPy:

* Hammer 4-point rule, alpha = (5 - sqrt 5)/20, beta = (5 + 3 sqrt 5)/20, w = 1/24
  (c3d10.py:21-32; the point *arrays* are what count, their comments do not match);
* shape-function derivatives through the volume coordinates (c3d10.py:35-106);
* J = dN/dxi . X, det J, inv J (c3d10.py:109-137);
* B (6 x 30) with engineering shears [gxy, gyz, gzx] (c3d10.py:140-189);
* isotropic C with G on the shear diagonal (c3d10.py:192-216);
* Ke = sum_g w B^T C B det J, then Ke = (Ke + Ke^T)/2 (c3d10.py:219-249);
* f_int = sum_g w B^T (C B u) det J (c3d10.py:252-283);
* Gauss-point stress and von Mises (c3d10.py:286-318).
"""

from __future__ import annotations

import numpy as np

ALPHA = (5.0 - np.sqrt(5.0)) / 20.0
BETA = (5.0 + 3.0 * np.sqrt(5.0)) / 20.0
WEIGHT = 1.0 / 24.0
GAUSS_POINTS = np.array(
    [[ALPHA, ALPHA, ALPHA], [BETA, ALPHA, ALPHA], [ALPHA, BETA, ALPHA], [ALPHA, ALPHA, BETA]], dtype=np.float64
)


def shape_functions(xi: float, eta: float, zeta: float):
    """N (10,) and dN/dxi (3, 10) at one natural point (c3d10.py:35-106)."""
    L1, L2, L3, L4 = 1.0 - xi - eta - zeta, xi, eta, zeta
    N = np.array(
        [
            L1 * (2 * L1 - 1),
            L2 * (2 * L2 - 1),
            L3 * (2 * L3 - 1),
            L4 * (2 * L4 - 1),
            4 * L1 * L2,
            4 * L2 * L3,
            4 * L3 * L1,
            4 * L1 * L4,
            4 * L2 * L4,
            4 * L3 * L4,
        ]
    )
    dL = np.zeros((4, 10))
    dL[0, [0, 4, 6, 7]] = [4 * L1 - 1, 4 * L2, 4 * L3, 4 * L4]
    dL[1, [1, 4, 5, 8]] = [4 * L2 - 1, 4 * L1, 4 * L3, 4 * L4]
    dL[2, [2, 5, 6, 9]] = [4 * L3 - 1, 4 * L2, 4 * L1, 4 * L4]
    dL[3, [3, 7, 8, 9]] = [4 * L4 - 1, 4 * L1, 4 * L2, 4 * L3]
    dN = np.stack([dL[1] - dL[0], dL[2] - dL[0], dL[3] - dL[0]])
    return N, dN


DN_DXI = np.stack([shape_functions(*gp)[1] for gp in GAUSS_POINTS])  # (4, 3, 10)


def elasticity_matrix(E: float, nu: float) -> np.ndarray:
    """6x6 isotropic C (c3d10.py:192-216)."""
    f = E / ((1.0 + nu) * (1.0 - 2.0 * nu))
    C = np.zeros((6, 6))
    C[:3, :3] = f * nu
    C[[0, 1, 2], [0, 1, 2]] = f * (1.0 - nu)
    C[[3, 4, 5], [3, 4, 5]] = E / (2.0 * (1.0 + nu))
    return C


def gauss_geometry(coords: np.ndarray):
    """Cartesian dN/dx (M, 4, 3, 10) and det J (M, 4) for coords (M, 10, 3).

    Raises like c3d10.py:129-134 on det J <= 0.
    """
    J = np.einsum("gkn,mnj->mgkj", DN_DXI, coords)  # (M,4,3,3)
    det = np.linalg.det(J)
    if np.any(det <= 0.0):
        bad = int(np.argmin(det.min(axis=1)))
        raise ValueError(f"Non-positive Jacobian determinant in C3D10 element {bad}")
    invJ = np.linalg.inv(J)
    dNdx = np.einsum("mgij,gjn->mgin", invJ, DN_DXI)
    return dNdx, det


def b_matrices(dNdx: np.ndarray) -> np.ndarray:
    """B (M, 4, 6, 30) from dN/dx (M, 4, 3, 10) (c3d10.py:166-187)."""
    M = dNdx.shape[0]
    B = np.zeros((M, 4, 6, 30))
    dx, dy, dz = dNdx[:, :, 0], dNdx[:, :, 1], dNdx[:, :, 2]
    B[:, :, 0, 0::3] = dx
    B[:, :, 1, 1::3] = dy
    B[:, :, 2, 2::3] = dz
    B[:, :, 3, 0::3] = dy
    B[:, :, 3, 1::3] = dx
    B[:, :, 4, 1::3] = dz
    B[:, :, 4, 2::3] = dy
    B[:, :, 5, 0::3] = dz
    B[:, :, 5, 2::3] = dx
    return B


def _c_batch(props: np.ndarray) -> np.ndarray:
    E, nu = props[:, 0], props[:, 1]
    f = E / ((1.0 + nu) * (1.0 - 2.0 * nu))
    C = np.zeros((len(E), 6, 6))
    C[:, :3, :3] = (f * nu)[:, None, None]
    for i in range(3):
        C[:, i, i] = f * (1.0 - nu)
        C[:, 3 + i, 3 + i] = E / (2.0 * (1.0 + nu))
    return C


def element_stiffness_batch(coords: np.ndarray, props: np.ndarray, chunk: int = 4096) -> np.ndarray:
    """Ke (M, 30, 30) for coords (M, 10, 3), props (M, 2) = [E, nu] (c3d10.py:219-249)."""
    M = coords.shape[0]
    out = np.empty((M, 30, 30))
    for s in range(0, M, chunk):
        c = coords[s : s + chunk]
        dNdx, det = gauss_geometry(c)
        B = b_matrices(dNdx)
        C = _c_batch(props[s : s + chunk])
        CB = np.einsum("mkl,mglj->mgkj", C, B)
        Ke = np.einsum("mg,mgki,mgkj->mij", WEIGHT * det, B, CB)
        out[s : s + chunk] = 0.5 * (Ke + Ke.transpose(0, 2, 1))
    return out


def element_internal_forces_batch(coords, u_e, props, chunk: int = 8192) -> np.ndarray:
    """f_int (M, 30) = sum_g w B^T C B u det J (c3d10.py:252-283)."""
    M = coords.shape[0]
    out = np.empty((M, 30))
    for s in range(0, M, chunk):
        dNdx, det = gauss_geometry(coords[s : s + chunk])
        B = b_matrices(dNdx)
        C = _c_batch(props[s : s + chunk])
        eps = np.einsum("mgij,mj->mgi", B, u_e[s : s + chunk])
        sig = np.einsum("mkl,mgl->mgk", C, eps)
        out[s : s + chunk] = np.einsum("mg,mgki,mgk->mi", WEIGHT * det, B, sig)
    return out


def element_stresses_batch(coords, u_e, props, chunk: int = 8192):
    """Gauss-point stresses (M, 4, 6) and von Mises (M, 4) (c3d10.py:286-318)."""
    M = coords.shape[0]
    sig_all = np.empty((M, 4, 6))
    for s in range(0, M, chunk):
        dNdx, _ = gauss_geometry(coords[s : s + chunk])
        B = b_matrices(dNdx)
        C = _c_batch(props[s : s + chunk])
        eps = np.einsum("mgij,mj->mgi", B, u_e[s : s + chunk])
        sig_all[s : s + chunk] = np.einsum("mkl,mgl->mgk", C, eps)
    sxx, syy, szz, sxy, syz, szx = np.moveaxis(sig_all, -1, 0)
    vm = np.sqrt(0.5 * ((sxx - syy) ** 2 + (syy - szz) ** 2 + (szz - sxx) ** 2 + 6.0 * (sxy**2 + syz**2 + szx**2)))
    return sig_all, vm
