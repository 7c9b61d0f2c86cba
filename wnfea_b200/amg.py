"""Smoothed-aggregation AMG of the C3D10 path: parameters, hierarchy export, host-only setup.

The hierarchy itself is built by the library (GPU setup with host aggregation by default, or
the whole setup in host C++; GPU apply).  This module
exposes its knobs (``AMGParams`` = ``wn_amg_params``) and reads a hierarchy back as scipy
matrices, for inspection and for the parity tests.  The reference's counterpart is the
beam-only ``BlockBeamAMGPreconditioner`` (wnfea/solver/amg_preconditioner.py:147-661);
its parameters map as: ``max_levels`` (:159), ``coarse_size`` (:159, in DOFs), the
Jacobi weight 0.67 (:449) is replaced by a Chebyshev smoother of ``smoother_degree`` (by default
degree 1: one Jacobi step before and one after the coarse correction, as the reference's V-cycle
takes (:504-536), weighted 1 / theta for the smoothing interval [lmax / 16, lmax]).  On the
6-DOF levels below the finest, ``coarse_block_smoother`` (default 1) makes that step block
Jacobi over each aggregate's 6 x 6 diagonal block: the GPU setup moves those levels to the
basis in which the diagonal blocks are the identity (A^ = T^T A T, T = diag(L_i^-T),
D_i = L_i L_i^T), where the point smoother is the block one; the exported levels are then
those of the new basis.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import call, ptr


@dataclass
class AMGParams:
    strength_theta: float = 0.08
    max_levels: int = 10
    coarse_size: int = 1500
    smoother_degree: int = 1
    cheb_lower: float = 1.0 / 16.0
    cheb_safety: float = 1.1
    prolong_omega: float = 4.0 / 3.0
    smooth_prolongator: int = 1
    power_iters: int = 15
    stream_min_mb: float = 4.0
    setup_on_device: int = 1
    coarse_block_smoother: int = 1

    def to_c(self) -> _lib.AmgParams:
        return _lib.AmgParams(**{f.name: getattr(self, f.name) for f in fields(self)})


def _bsr_export(fn, handle, level, which):
    br, bc = C.c_int(), C.c_int()
    nr, nc, nb = C.c_int64(), C.c_int64(), C.c_int64()
    call(fn, handle, level, which, C.byref(br), C.byref(bc), C.byref(nr), C.byref(nc), C.byref(nb), None, None, None)
    rp = np.empty(nr.value + 1, dtype=np.int32)
    ci = np.empty(nb.value, dtype=np.int32)
    v = np.empty((nb.value, br.value, bc.value))
    call(fn, handle, level, which, C.byref(br), C.byref(bc), C.byref(nr), C.byref(nc), C.byref(nb), ptr(rp), ptr(ci),
         ptr(v))
    return sp.bsr_matrix((v, ci, rp), shape=(nr.value * br.value, nc.value * bc.value))


@dataclass
class HierarchyLevel:
    bs: int
    n_nodes: int
    rho: float
    dinv: np.ndarray
    A: sp.bsr_matrix | None  # None for level 0 (the assembled matrix)
    P: sp.bsr_matrix
    R: sp.bsr_matrix


@dataclass
class Hierarchy:
    levels: list[HierarchyLevel]
    coarse_A: np.ndarray
    coarse_inv: np.ndarray


def export_system_hierarchy(system) -> Hierarchy:
    """The hierarchy of a ``SolidSystem`` after ``wn_amg_setup``."""
    h = system.handle
    nl = C.c_int()
    bs = (C.c_int * 16)()
    nn = (C.c_int64 * 16)()
    call("wn_amg_info", h, C.byref(nl), bs, nn, None, None, None)
    levels = []
    for lvl in range(nl.value - 1):
        n = nn[lvl] * bs[lvl]
        dinv = np.empty(n)
        rho = C.c_double()
        call("wn_amg_level_data", h, lvl, C.byref(rho), ptr(dinv))
        A = None if lvl == 0 else _bsr_export("wn_amg_level_matrix", h, lvl, 0)
        levels.append(HierarchyLevel(bs[lvl], nn[lvl], rho.value, dinv, A,
                                     _bsr_export("wn_amg_level_matrix", h, lvl, 1),
                                     _bsr_export("wn_amg_level_matrix", h, lvl, 2)))
    nc = C.c_int64()
    call("wn_amg_coarse", h, C.byref(nc), None, None)
    Ac = np.empty((nc.value, nc.value))
    Ai = np.empty((nc.value, nc.value))
    call("wn_amg_coarse", h, C.byref(nc), ptr(Ac), ptr(Ai))
    return Hierarchy(levels, Ac, Ai)


def setup_host(K_bsr3: sp.bsr_matrix, coords: np.ndarray, fixed_mask: np.ndarray | None = None,
               params: AMGParams | None = None) -> Hierarchy:
    """Run the library's AMG setup on the host only (no GPU) and export the hierarchy."""
    K = sp.bsr_matrix(K_bsr3, blocksize=(3, 3))
    K.sort_indices()
    rp = np.ascontiguousarray(K.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(K.indices, dtype=np.int32)
    v = np.ascontiguousarray(K.data, dtype=np.float64)
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    fm = None if fixed_mask is None else np.ascontiguousarray(fixed_mask, dtype=np.uint8)
    prm = (params or AMGParams()).to_c()
    out = C.c_void_p()
    call("wn_amg_setup_host", len(rp) - 1, ptr(rp), ptr(ci), ptr(v), ptr(coords), ptr(fm), C.byref(prm), C.byref(out))
    try:
        nlev = C.c_int64()
        call("wn_amg_host_level_data", out, -1, None, None, C.byref(nlev), None)
        levels = []
        for lvl in range(nlev.value):
            nn, bs, rho = C.c_int64(), C.c_int(), C.c_double()
            call("wn_amg_host_level_data", out, lvl, None, None, C.byref(nn), C.byref(bs))
            dinv = np.empty(nn.value * bs.value)
            call("wn_amg_host_level_data", out, lvl, C.byref(rho), ptr(dinv), C.byref(nn), C.byref(bs))
            A = None if lvl == 0 else _bsr_export("wn_amg_host_level_matrix", out, lvl, 0)
            levels.append(HierarchyLevel(bs.value, nn.value, rho.value, dinv, A,
                                         _bsr_export("wn_amg_host_level_matrix", out, lvl, 1),
                                         _bsr_export("wn_amg_host_level_matrix", out, lvl, 2)))
        nc = C.c_int64()
        call("wn_amg_host_coarse", out, C.byref(nc), None, None)
        Ac = np.empty((nc.value, nc.value))
        Ai = np.empty((nc.value, nc.value))
        call("wn_amg_host_coarse", out, C.byref(nc), ptr(Ac), ptr(Ai))
        return Hierarchy(levels, Ac, Ai)
    finally:
        _lib.lib().wn_amg_host_destroy(out)
