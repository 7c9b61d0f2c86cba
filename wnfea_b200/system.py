"""Device-resident C3D10 system (handle around ``wn_solid_*``) and the BSR3 matrix object.

``SolidSystem`` owns one library handle: the mesh, the 3x3-block pattern, the element ->
block map, the assembled FP64/FP32 values and the Dirichlet mask, all on the GPU.
``BSR3Matrix`` is what ``assemble_c3d10_sparse_3dof`` returns in place of the reference's
scipy CSR (solid_solver.py:26-129): it keeps ``.shape``/``.nnz`` and converts with
``.tocsr()`` / ``.to_bsr()`` for comparisons with scipy.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import call, ptr


class SolidSystem:
    """One C3D10 mesh on the GPU (nodes (N,3) float64, conn (M,10) int)."""

    def __init__(self, nodes: np.ndarray, conn: np.ndarray):
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        if self.nodes.ndim != 2 or self.nodes.shape[1] != 3:
            raise ValueError("nodes must have shape (N, 3)")
        if self.conn.ndim != 2 or self.conn.shape[1] != 10:
            raise ValueError("conn must have shape (M, 10)")
        h = C.c_void_p()
        call("wn_solid_create", len(self.nodes), len(self.conn), ptr(self.nodes), ptr(self.conn), C.byref(h))
        self._h = h
        n, m, b = C.c_int64(), C.c_int64(), C.c_int64()
        call("wn_solid_info", self._h, C.byref(n), C.byref(m), C.byref(b))
        self.n_nodes, self.n_el, self.nnzb = n.value, m.value, b.value
        self.fixed_mask = np.zeros(3 * self.n_nodes, dtype=np.uint8)
        self.props: np.ndarray | None = None
        self.bcs_applied = False
        self.amg_ready = False

    # -- lifetime -------------------------------------------------------------------------
    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            try:
                _lib.lib().wn_solid_destroy(self._h)
            finally:
                self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- pattern ----------------------------------------------------------------------------
    def pattern(self) -> tuple[np.ndarray, np.ndarray]:
        rp = np.empty(self.n_nodes + 1, dtype=np.int32)
        ci = np.empty(self.nnzb, dtype=np.int32)
        call("wn_solid_get_pattern", self._h, ptr(rp), ptr(ci))
        return rp, ci

    def element_map(self) -> np.ndarray:
        m = np.empty((self.n_el, 100), dtype=np.int32)
        call("wn_solid_get_map", self._h, ptr(m))
        return m

    def set_streaming(self, enable: bool, batched: bool = False) -> None:
        """Streamed fine-level kernels (tile-major packs, the default for single-case solves) on or
        off; off frees the packs (about 1 GB per million DOFs) and runs the fine level on the
        register row kernels.  ``batched`` streams the fine level of the 32-case solves too (they
        default to the register kernels)."""
        call("wn_solid_set_stream", self._h, (2 if batched else 1) if enable else 0)

    def set_batch_staging(self, enable: bool) -> None:
        """Batched solves: the FP32 fine-level passes with each row tile's x slice staged in
        shared memory, or the register row kernels gathering x through the caches (the default,
        faster on the 1M-DOF I-beam); bitwise the same row products."""
        call("wn_solid_set_batch_staging", self._h, int(bool(enable)))

    # -- assembly ---------------------------------------------------------------------------
    def set_fixed(self, fixed_dofs) -> None:
        mask = np.zeros(3 * self.n_nodes, dtype=np.uint8)
        if fixed_dofs is not None and len(fixed_dofs):
            mask[np.asarray(fixed_dofs, dtype=np.int64)] = 1
        self.fixed_mask = mask
        call("wn_solid_set_fixed", self._h, ptr(mask))

    def assemble(self, props: np.ndarray, apply_bcs: bool = True) -> None:
        props = np.ascontiguousarray(props, dtype=np.float64)
        if props.shape != (self.n_el, 2):
            raise ValueError(f"props must have shape ({self.n_el}, 2)")
        call("wn_assemble_c3d10", self._h, ptr(props), int(bool(apply_bcs)))
        self.props = props
        self.bcs_applied = bool(apply_bcs)
        self.amg_ready = False

    # -- solver -------------------------------------------------------------------------------
    def amg_setup(self, params=None) -> None:
        from .amg import AMGParams

        prm = (params or AMGParams()).to_c()
        call("wn_amg_setup", self._h, C.byref(prm))
        self.amg_ready = True

    def solve(self, F: np.ndarray, rtol: float = 1e-8, max_iter: int = 2000, precond: int = 2,
              precision: int = 0, inner_rtol: float = 0.0, max_outer: int = 10, chunk: int = 8,
              use_graph: bool = True, profile: bool = False):
        """Solve K u = F on the GPU (host buffers); returns (u, stats dict).  ``profile``: time
        every kernel with CUDA events (read back with ``profile_table()``)."""
        F = np.ascontiguousarray(F, dtype=np.float64)
        u = np.empty_like(F)
        prm = _lib.SolveParams(rtol, max_iter, precond, precision, inner_rtol, max_outer, chunk, int(use_graph),
                               int(profile))
        st = _lib.SolveStats()
        call("wn_solve", self._h, ptr(F), ptr(u), C.byref(prm), C.byref(st))
        return u, {f: getattr(st, f) for f, _ in _lib.SolveStats._fields_}

    def profile_table(self) -> dict:
        """{kernel class: (launches, ms, algorithmic bytes)} of the last profiled solve."""
        n = C.c_int()
        call("wn_solve_profile", self._h, 0, C.byref(n), None, None, None, None)
        k = n.value
        names = C.create_string_buffer(48 * max(k, 1))
        counts = np.zeros(k, dtype=np.int64)
        ms = np.zeros(k)
        by = np.zeros(k)
        call("wn_solve_profile", self._h, k, C.byref(n), names, ptr(counts), ptr(ms), ptr(by))
        raw = names.raw
        return {raw[48 * i:48 * i + 48].split(b"\0", 1)[0].decode(): (int(counts[i]), float(ms[i]), float(by[i]))
                for i in range(k)}

    def solve_multi(self, F: np.ndarray, rtol: float = 1e-8, max_iter: int = 2000, precond: int = 2,
                    precision: int = 1, max_outer: int = 10, chunk: int = 8, use_graph: bool = True):
        """Solve K U = F for the load cases in the columns of F (n x k, host) in batches of 32
        sharing every matrix read; returns (U, stats dict with per-case 'case_iterations' and
        'case_rel_res')."""
        F = np.ascontiguousarray(F, dtype=np.float64)
        if F.ndim == 1:
            F = F[:, None]
        k = F.shape[1]
        U = np.empty_like(F)
        prm = _lib.SolveParams(rtol, max_iter, precond, precision, 0.0, max_outer, chunk, int(use_graph))
        st = _lib.SolveStats()
        its = np.zeros(k, dtype=np.int32)
        rel = np.zeros(k)
        call("wn_solve_multi", self._h, k, ptr(F), ptr(U), C.byref(prm), C.byref(st), ptr(its), ptr(rel))
        out = {f: getattr(st, f) for f, _ in _lib.SolveStats._fields_}
        out["case_iterations"] = its
        out["case_rel_res"] = rel
        return U, out

    def solve_multi_device(self, F, U, rtol: float = 1e-8, max_iter: int = 2000, precond: int = 2,
                           precision: int = 1, max_outer: int = 10, chunk: int = 8, stream: int = 0):
        """Device-pointer variant: F, U are CUDA tensors of shape (n, k), row-major, float64."""
        k = int(F.shape[1])
        prm = _lib.SolveParams(rtol, max_iter, precond, precision, 0.0, max_outer, chunk, 1)
        st = _lib.SolveStats()
        its = np.zeros(k, dtype=np.int32)
        rel = np.zeros(k)
        call("wn_solve_multi_device", self._h, k, _lib.dptr(F), _lib.dptr(U), C.byref(prm), C.byref(st), ptr(its),
             ptr(rel), stream)
        out = {f: getattr(st, f) for f, _ in _lib.SolveStats._fields_}
        out["case_iterations"] = its
        out["case_rel_res"] = rel
        return out

    def matvec(self, x: np.ndarray) -> np.ndarray:
        rp, ci = self.pattern()
        v = self.values()
        y = np.zeros(3 * self.n_nodes)
        call("wn_spmv_bsr_f64", 3, 3, self.n_nodes, self.n_nodes, self.nnzb, ptr(rp), ptr(ci), ptr(v),
             ptr(np.ascontiguousarray(x, dtype=np.float64)), ptr(y), 1.0, 0.0)
        return y

    def values(self) -> np.ndarray:
        v = np.empty((self.nnzb, 3, 3), dtype=np.float64)
        call("wn_solid_get_values", self._h, ptr(v))
        return v

    # -- element-level operators --------------------------------------------------------------
    def internal_forces(self, u: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        f = np.empty(3 * self.n_nodes)
        call("wn_fint_c3d10", self._h, ptr(u), ptr(f))
        return f

    def stress_field(self, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        sig = np.empty((self.n_el, 6))
        vm = np.empty(self.n_el)
        nvm = np.empty(self.n_nodes)
        call("wn_stress_c3d10", self._h, ptr(u), ptr(sig), ptr(vm), ptr(nvm))
        return sig, vm, nvm

    def compliance_gradient(self, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        gE = np.empty(self.n_el)
        gF = np.empty(3 * self.n_nodes)
        call("wn_adjoint_compliance", self._h, ptr(u), ptr(gE), ptr(gF))
        return gE, gF


class BSR3Matrix:
    """The assembled stiffness matrix, resident on the GPU in 3x3-block BSR form."""

    def __init__(self, system: SolidSystem):
        self.system = system

    @property
    def shape(self) -> tuple[int, int]:
        n = 3 * self.system.n_nodes
        return (n, n)

    @property
    def nnz_blocks(self) -> int:
        return self.system.nnzb

    @property
    def nnz(self) -> int:
        """Stored scalar entries (9 per block, Dirichlet zeros included)."""
        return 9 * self.system.nnzb

    @property
    def dtype(self):
        return np.dtype(np.float64)

    def to_bsr(self) -> sp.bsr_matrix:
        rp, ci = self.system.pattern()
        return sp.bsr_matrix((self.system.values(), ci, rp), shape=self.shape)

    def tocsr(self) -> sp.csr_matrix:
        """Scalar CSR; with BCs applied, explicit zeros are dropped as eliminate_zeros does
        (solid_solver.py:127)."""
        K = self.to_bsr().tocsr()
        K.sort_indices()
        if self.system.bcs_applied:
            K.eliminate_zeros()
        return K

    def diagonal(self) -> np.ndarray:
        return self.tocsr().diagonal()

    def __matmul__(self, x):
        return self.system.matvec(np.asarray(x, dtype=np.float64))
