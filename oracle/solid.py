"""ORACLE (test infrastructure only) -- FP64 CPU restatement of the reference's C3D10 solve path.

Nothing in the product imports this module.  Tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it as the checker.

Follows wnfea/solver/solid_solver.py:

* ``assemble``            -- assemble_c3d10_sparse_3dof (solid_solver.py:26-129): 30-DOF
                             node-major template, COO -> CSR duplicate summation, loads,
                             FIXED translational DOFs, row/col zeroing, diag = 1, F = 0,
                             eliminate_zeros;
* ``pcg``                 -- solve_c3d10_pcg (solid_solver.py:197-308): Jacobi / 3x3
                             block-Jacobi / none, FP64 scipy ``cg``; mixed_fp32 iterative
                             refinement with <= 10 outer FP64 residuals (the iteration count
                             returned here is the real count -- the reference stores scipy's
                             ``info`` there, solid_solver.py:288-291);
* ``stress_field``        -- compute_c3d10_stress_field (solid_solver.py:311-365);
* ``bsr3_pattern_and_map``-- the 3x3-block pattern of the same matrix, and for every element
                             and local node pair (a, b) the index of block
                             (conn[e,a], conn[e,b]); new (the reference stores scalar CSR), so
                             it is pinned against the CSR pattern above (nnz == 9 * nnzb);
* ``compliance_gradient`` -- dC/dE_e = -u_e^T Ke u_e / E_e, dC/dF = 2u (free DOFs); new.
"""

from __future__ import annotations

import time

import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import LinearOperator, cg

from . import c3d10


def element_dofs(conn: np.ndarray) -> np.ndarray:
    """(M, 30) global DOF indices, node-major [ux, uy, uz] (solid_solver.py:55-60)."""
    return (conn[:, :, None].astype(np.int64) * 3 + np.arange(3)).reshape(len(conn), 30)


def assemble(nodes, conn, props, F_loads=None, fixed_dofs=None, apply_bcs=True, Ke=None):
    """K (CSR), F, fixed_dofs exactly as assemble_c3d10_sparse_3dof does it."""
    n_dofs = 3 * len(nodes)
    if Ke is None:
        Ke = c3d10.element_stiffness_batch(nodes[conn], props)
    dofs = element_dofs(conn)
    rows = np.repeat(dofs, 30, axis=1).ravel()
    cols = np.tile(dofs, (1, 30)).ravel()
    K = sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(n_dofs, n_dofs)).tocsr()
    F = np.zeros(n_dofs) if F_loads is None else np.array(F_loads, dtype=np.float64)
    fixed = [] if fixed_dofs is None else [int(d) for d in fixed_dofs]
    if apply_bcs and len(fixed):
        apply_dirichlet(K, F, fixed)
    return K, F, fixed


def apply_dirichlet(K: sp.csr_matrix, F: np.ndarray, fixed) -> None:
    """In-place BCs of solid_solver.py:105-127 (off-diagonals zeroed, diag = 1, F = 0)."""
    n = K.shape[0]
    is_fixed = np.zeros(n, dtype=bool)
    is_fixed[np.asarray(list(fixed), dtype=np.int64)] = True
    row = np.repeat(np.arange(n), np.diff(K.indptr))
    mr, mc = is_fixed[row], is_fixed[K.indices]
    K.data[(mr | mc) & (row != K.indices)] = 0.0
    K.data[mr & (row == K.indices)] = 1.0
    F[is_fixed] = 0.0
    K.eliminate_zeros()


def pcg(K, F, rtol=1e-6, max_iter=2000, preconditioner="jacobi", precision="fp64"):
    """(u, iterations, final_rel_res, seconds) like solve_c3d10_pcg (solid_solver.py:197-308)."""
    t0 = time.perf_counter()
    n = K.shape[0]
    d = K.diagonal()
    dinv = np.where(np.abs(d) > 1e-12, 1.0 / d, 1.0)
    if preconditioner == "jacobi":
        M = LinearOperator((n, n), matvec=lambda v: dinv * v, dtype=np.float64)
    elif preconditioner == "block_jacobi":
        blocks = np.zeros((n // 3, 3, 3))
        for i in range(3):
            for j in range(3):
                blocks[:, i, j] = np.asarray(K[np.arange(i, n, 3), np.arange(j, n, 3)]).ravel()
        inv = np.linalg.pinv(blocks)
        M = LinearOperator((n, n), matvec=lambda v: np.matmul(inv, v.reshape(-1, 3, 1)).ravel(), dtype=np.float64)
    else:
        M = None
    nb = float(np.linalg.norm(F))
    if nb == 0.0:
        return np.zeros(n), 0, 0.0, 0.0
    count = [0]

    def cb(_):
        count[0] += 1

    if precision == "mixed_fp32":
        K32 = K.astype(np.float32)
        d32 = dinv.astype(np.float32)
        P32 = LinearOperator((n, n), matvec=lambda v: d32 * v, dtype=np.float32)
        u = np.zeros(n)
        r = F - K @ u
        for _ in range(10):
            if np.linalg.norm(r) / nb < rtol:
                break
            du, _info = cg(K32, r.astype(np.float32), M=P32, rtol=max(1e-4, rtol), maxiter=max_iter // 5, callback=cb)
            u += du.astype(np.float64)
            r = F - K @ u
        return u, count[0], float(np.linalg.norm(r) / nb), time.perf_counter() - t0
    u, _info = cg(K, F, M=M, rtol=rtol, maxiter=max_iter, callback=cb)
    r = F - K @ u
    return u, count[0], float(np.linalg.norm(r) / nb), time.perf_counter() - t0


def stress_field(nodes, conn, props, u):
    """cell stresses (M, 6), cell von Mises (M,), nodal von Mises (n,) (solid_solver.py:311-365)."""
    u_e = u.reshape(-1, 3)[conn].reshape(len(conn), 30)
    sig, vm = c3d10.element_stresses_batch(nodes[conn], u_e, props)
    cell_sig = sig.mean(axis=1)
    cell_vm = vm.mean(axis=1)
    n = len(nodes)
    acc = np.zeros(n)
    cnt = np.zeros(n, dtype=np.int64)
    np.add.at(acc, conn.ravel(), np.repeat(cell_vm, 10))
    np.add.at(cnt, conn.ravel(), 1)
    nodal = np.zeros(n)
    m = cnt > 0
    nodal[m] = acc[m] / cnt[m]
    return cell_sig, cell_vm, nodal


def bsr3_pattern_and_map(conn: np.ndarray, n_nodes: int):
    """Sorted 3x3-block pattern (row_ptr, col_idx) and the (M, 100) element->block map.

    Block (i, j) exists iff nodes i and j share an element; columns are sorted within a
    row; map[e, 10 a + b] = index of block (conn[e, a], conn[e, b]).
    """
    M = len(conn)
    r = np.repeat(conn, 10, axis=1).astype(np.int64).ravel()
    c = np.tile(conn, (1, 10)).astype(np.int64).ravel()
    key = r * n_nodes + c
    uniq, inv = np.unique(key, return_inverse=True)
    rows = uniq // n_nodes
    cols = (uniq % n_nodes).astype(np.int32)
    row_ptr = np.zeros(n_nodes + 1, dtype=np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    emap = inv.reshape(M, 100).astype(np.int32)
    return row_ptr, cols, emap


def bsr3_from_csr(K: sp.csr_matrix, row_ptr, col_idx) -> np.ndarray:
    """Values (nnzb, 3, 3) of the scalar CSR ``K`` on the given block pattern."""
    n_nodes = len(row_ptr) - 1
    rows = np.repeat(np.arange(n_nodes), np.diff(row_ptr))
    vals = np.zeros((len(col_idx), 3, 3))
    Kc = K.tocsr()
    for a in range(3):
        for b in range(3):
            vals[:, a, b] = np.asarray(Kc[rows * 3 + a, col_idx.astype(np.int64) * 3 + b]).ravel()
    return vals


def bsr3_to_csr(row_ptr, col_idx, vals, eliminate_zeros=False) -> sp.csr_matrix:
    """Scalar CSR from a 3x3-block matrix (for comparisons against the reference CSR)."""
    n_nodes = len(row_ptr) - 1
    B = sp.bsr_matrix((np.asarray(vals).reshape(-1, 3, 3), col_idx, row_ptr), shape=(3 * n_nodes, 3 * n_nodes))
    K = B.tocsr()
    K.sort_indices()
    if eliminate_zeros:
        K.eliminate_zeros()
    return K


def compliance_gradient(nodes, conn, props, u, fixed_mask=None):
    """dC/dE_e = -u_e^T Ke u_e / E_e and dC/dF = 2u (0 on fixed DOFs) for C = F^T u."""
    u_e = u.reshape(-1, 3)[conn].reshape(len(conn), 30)
    f = c3d10.element_internal_forces_batch(nodes[conn], u_e, props)
    gE = -np.einsum("mi,mi->m", u_e, f) / props[:, 0]
    gF = 2.0 * u
    if fixed_mask is not None:
        gF = np.where(fixed_mask, 0.0, gF)
    return gE, gF
