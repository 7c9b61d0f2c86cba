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
* PCG with the V-cycle as M^-1 (nonlinear_solver.py:51-156 structure);
* optionally block-Jacobi smoothing on the 6-DOF levels (``block_rho``), the smoother the
  library's coarse-level change of basis yields (no reference counterpart: the reference's
  V-cycle smooths with point Jacobi, amg_preconditioner.py:447-454).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


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
    """Chebyshev steps; dinv is the point-Jacobi vector or a (block-diagonal) matrix."""
    apply = (lambda v: dinv * v) if isinstance(dinv, np.ndarray) else (lambda v: dinv @ v)
    r = apply(b - A @ x)
    d = r * inv_theta
    x = x + d
    for k in range(len(c1)):
        r = r - apply(A @ d)
        d = c1[k] * d + c2[k] * r
        x = x + d
    return x


def diag_blocks(A, bs):
    """The bs x bs diagonal blocks of A, shape (n, bs, bs)."""
    A = sp.csr_matrix(A)
    n = A.shape[0] // bs
    idx = np.arange(n) * bs
    return np.stack([np.stack([A[idx + r, idx + c].A1 for c in range(bs)], axis=1) for r in range(bs)], axis=1)


def block_cholesky(D, pivot_tol=1e-13):
    """Lower Cholesky factors of the blocks D (n, bs, bs), with the library's rule for a
    direction a block does not span: a pivot at or below pivot_tol x the block's largest
    diagonal entry becomes 1, with that row and column of L zeroed (the DOF keeps its basis)."""
    n, bs, _ = D.shape
    L = np.zeros_like(D)
    scale = np.abs(np.diagonal(D, axis1=1, axis2=2)).max(axis=1)
    for c in range(bs):
        d = D[:, c, c] - np.sum(L[:, c, :c] ** 2, axis=1)
        ok = d > pivot_tol * scale
        dc = np.sqrt(np.where(ok, d, 1.0))
        L[:, c, :c] = np.where(ok[:, None], L[:, c, :c], 0.0)
        L[:, c, c] = dc
        for r in range(c + 1, bs):
            sr = D[:, r, c] - np.sum(L[:, r, :c] * L[:, c, :c], axis=1)
            L[:, r, c] = np.where(ok, sr / dc, 0.0)
    return L


def block_diag_inverse(A, bs):
    """The block-Jacobi smoother of A: the block-diagonal (L_i L_i^T)^-1 with L_i the factor of
    diagonal block i (``block_cholesky``; D_i^-1 where D_i is positive definite)."""
    Li = np.linalg.inv(block_cholesky(diag_blocks(A, bs)))
    n = Li.shape[0]
    Binv = np.einsum("nji,njk->nik", Li, Li)  # L^-T L^-1
    return sp.bsr_matrix((Binv, np.arange(n), np.arange(n + 1)), shape=A.shape).tocsr()


def vcycle(K0, hier, b, degree=1, level=0, dtype=np.float64, lower=1.0 / 16.0, safety=1.1, block_rho=None):
    """z = M^-1 b for the exported hierarchy; all arithmetic in ``dtype``.

    block_rho: None (point Jacobi everywhere, as exported), or per level l >= 1 the estimate of
    rho(D_block^-1 A_l): those levels are then smoothed with 6 x 6 block Jacobi on the exported
    (point-basis) matrices -- the smoother the library's coarse-level change of basis yields."""
    if level == len(hier.levels):
        return (hier.coarse_inv @ b.astype(np.float64)).astype(dtype)
    L = hier.levels[level]
    A = (K0 if level == 0 else L.A).astype(dtype)
    rho = L.rho
    if block_rho is not None and level >= 1:
        dinv = block_diag_inverse(L.A, L.bs).astype(dtype)
        rho = block_rho[level]
    else:
        dinv = L.dinv.astype(dtype)
    it, c1, c2 = cheb_coefficients(rho, degree, lower, safety)
    it = dtype(it)
    c1 = [dtype(c) for c in c1]
    c2 = [dtype(c) for c in c2]
    b = b.astype(dtype)
    x = _cheb(A, dinv, b, np.zeros_like(b), it, c1, c2)
    res = b - A @ x
    bc = L.R.astype(dtype) @ res
    xc = vcycle(K0, hier, bc, degree, level + 1, dtype, lower, safety, block_rho)
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
