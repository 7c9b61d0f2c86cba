"""ORACLE (test infrastructure only) -- FP64/FP32 CPU restatement of the AMG V-cycle and PCG.

Nothing in the product imports this module.  Given a hierarchy exported from the library
(level matrices, 1/diag, spectral radius estimates, the dense coarsest inverse), it applies
the V-cycle exactly as the GPU kernels are specified:

* recursive V-cycle structure of the reference (amg_preconditioner.py:504-536): pre-smooth
  from a zero guess, residual, restrict with R = P^T, coarse correction, prolongate,
  post-smooth; the coarsest level is a dense Cholesky solve (:309-325), here applied as
  the explicit inverse L^-T L^-1;
* smoother: Chebyshev polynomial in D^-1 A on [lower * lmax, lmax], lmax = safety * rho
  (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 12.1), in place of the
  reference's Jacobi weight 0.67 (:447-454);
* PCG with the V-cycle as M^-1 (nonlinear_solver.py:51-156 structure).
"""

from __future__ import annotations

import numpy as np


def cheb_coefficients(rho, degree, lower=1.0 / 16.0, safety=1.1):
    lmax = safety * rho
    lmin = lower * lmax
    theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
    sigma = theta / delta
    r_old = 1.0 / sigma
    c1, c2 = [], []
    for _ in range(1, degree):
        r_new = 1.0 / (2.0 * sigma - r_old)
        c1.append(r_new * r_old)
        c2.append(2.0 * r_new / delta)
        r_old = r_new
    return 1.0 / theta, c1, c2


def _cheb(A, dinv, b, x, inv_theta, c1, c2):
    r = dinv * (b - A @ x)
    d = r * inv_theta
    x = x + d
    for k in range(len(c1)):
        r = r - dinv * (A @ d)
        d = c1[k] * d + c2[k] * r
        x = x + d
    return x


def vcycle(K0, hier, b, degree=1, level=0, dtype=np.float64, lower=1.0 / 16.0, safety=1.1):
    """z = M^-1 b for the exported hierarchy; all arithmetic in ``dtype``."""
    if level == len(hier.levels):
        return (hier.coarse_inv @ b.astype(np.float64)).astype(dtype)
    L = hier.levels[level]
    A = (K0 if level == 0 else L.A).astype(dtype)
    dinv = L.dinv.astype(dtype)
    it, c1, c2 = cheb_coefficients(L.rho, degree, lower, safety)
    it = dtype(it)
    c1 = [dtype(c) for c in c1]
    c2 = [dtype(c) for c in c2]
    b = b.astype(dtype)
    x = _cheb(A, dinv, b, np.zeros_like(b), it, c1, c2)
    res = b - A @ x
    bc = L.R.astype(dtype) @ res
    xc = vcycle(K0, hier, bc, degree, level + 1, dtype, lower, safety)
    x = x + L.P.astype(dtype) @ xc
    return _cheb(A, dinv, b, x, it, c1, c2)


def pcg(K, F, M, rtol=1e-8, max_iter=1000):
    """Preconditioned CG; stops on the recursive residual like the GPU solver."""
    x = np.zeros_like(F)
    r = F.copy()
    z = M(r)
    p = z.copy()
    rz = r @ z
    nb = np.linalg.norm(F)
    for it in range(max_iter):
        q = K @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if np.linalg.norm(r) <= rtol * nb:
            return x, it + 1
        z = M(r)
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, max_iter
