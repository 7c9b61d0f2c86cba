"""C3D10 solid solve path with the reference's API (wnfea/solver/solid_solver.py).

* ``assemble_c3d10_sparse_3dof(model, apply_bcs=True) -> (K, F, fixed_dofs)``
  (solid_solver.py:26-129): K is a GPU-resident ``BSR3Matrix`` (``.shape``, ``.nnz``,
  ``.tocsr()``, ``.to_bsr()``), assembled by the sm_100a element kernel through the
  atomic-free element -> block map;
* ``solve_c3d10_system(K, F, method, rtol, max_iter, preconditioner, precision)
  -> (u, stats)`` (solid_solver.py:132-194);
* ``solve_c3d10_pcg(K, F, rtol, max_iter, preconditioner, precision)
  -> (u, iterations, final_rel_res, solve_time_sec)`` (solid_solver.py:197-308);
* ``compute_c3d10_stress_field(model, u) -> (cell_stresses, cell_vm, nodal_vm)``
  (solid_solver.py:311-365).

Every computation runs on the GPU through libwnfea_cuda; there is no CPU fallback.
"""

from __future__ import annotations

import time

import numpy as np

from .model import FEAModel, solid_element_props, solid_fixed_dofs, solid_load_vector
from .system import BSR3Matrix, SolidSystem


def _mesh_key(model: FEAModel):
    n, c = model.mesh_nodes, model.solid_elements
    return (id(n), n.shape, id(c), c.shape)


def solid_system(model: FEAModel) -> SolidSystem:
    """The model's GPU system, created once per mesh and cached on the model."""
    key = _mesh_key(model)
    cached = getattr(model, "_wn_system", None)
    if cached is not None and cached[0] == key:
        return cached[1]
    sysobj = SolidSystem(model.mesh_nodes, model.solid_elements)
    object.__setattr__(model, "_wn_system", (key, sysobj))
    return sysobj


def assemble_c3d10_sparse_3dof(model: FEAModel, apply_bcs: bool = True):
    """Assemble K (GPU BSR3), F and the fixed DOF list exactly as solid_solver.py:26-129."""
    if model.mesh_nodes is None or model.solid_elements is None:
        raise ValueError("model has no C3D10 mesh")
    system = solid_system(model)
    F = solid_load_vector(model)
    fixed = [int(d) for d in solid_fixed_dofs(model)] if (apply_bcs and model.supports) else []
    system.set_fixed(fixed)
    system.assemble(solid_element_props(model), apply_bcs=bool(apply_bcs and fixed))
    if fixed:
        F[np.asarray(fixed, dtype=np.int64)] = 0.0
    return BSR3Matrix(system), F, fixed


_PRECOND = {"none": 0, "jacobi": 1, "amg": 2, "block_jacobi": 3}
_PRECISION = {"fp64": 0, "mixed_fp32": 1, "mixed_fp32_ir": 2, "mixed_fp16": 3}


def solve_c3d10_pcg(
    K: BSR3Matrix,
    F: np.ndarray,
    rtol: float = 1e-6,
    max_iter: int = 2000,
    preconditioner: str = "jacobi",
    precision: str = "fp64",
    amg_params=None,
    inner_rtol: float = 0.0,
    chunk: int = 8,
):
    """PCG on the GPU -> (u, iterations, final_rel_res, solve_time_sec) (solid_solver.py:197-308).

    Defaults are the reference's (rtol 1e-6, 2000 iterations, point Jacobi, FP64).
    ``preconditioner``: "jacobi" (point Jacobi, :228-236), "block_jacobi" (pseudo-inverse of
    every 3x3 node block, :237-258), "none", or "amg" (smoothed-aggregation AMG V-cycle; no
    reference counterpart for solids, and the fast choice for large meshes).  ``precision``:

    * "fp64"          -- FP64 matrix, vectors, dots and preconditioner;
    * "mixed_fp32"    -- FP64 PCG (FP64 SpMV, x, r, q and dots; FP32 search directions on the
                         streamed fine level) with the preconditioner in FP32
                         (for "amg": FP32 V-cycle values, vectors and accumulation, FP64
                         coarsest inverse), inside the FP64 true-residual loop;
    * "mixed_fp32_ir" -- the scheme of the reference's mixed mode (:271-300): FP32 PCG (FP32
                         SpMV, FP32 preconditioner, FP64 dots) inside FP64 iterative
                         refinement.  Converges slowly once cond(K) * 6e-8 approaches 1 (an
                         FP32 SpMV cannot resolve smooth displacement fields: K u cancels ~8
                         digits per row); fine for small meshes;
    * "mixed_fp16"    -- "mixed_fp32" with the V-cycle's fine level on the equilibrated matrix
                         S K S (S = diag(K)^-1/2, entries in [-1, 1]) stored in FP16, FP32
                         arithmetic and vectors: the FP16 preconditioner of the reference's
                         TRI_PRECISION (mixed_precision.py:96-103), on every iteration.  "amg"
                         only.

    All modes stop on the true FP64 residual ||F - K u|| <= rtol ||F||.  The returned
    iteration count is the real one (the reference stores scipy's ``info`` there,
    :288-291).
    """
    if preconditioner not in _PRECOND:
        raise ValueError(f"preconditioner must be one of {sorted(_PRECOND)}, got {preconditioner!r}")
    if precision not in _PRECISION:
        raise ValueError(f"precision must be one of {sorted(_PRECISION)}, got {precision!r}")
    if precision == "mixed_fp16" and preconditioner != "amg":
        raise ValueError("precision 'mixed_fp16' (FP16 V-cycle) needs preconditioner='amg'")
    t0 = time.perf_counter()
    system = K.system
    if preconditioner == "amg" and (amg_params is not None or not system.amg_ready):
        system.amg_setup(amg_params)
    u, st = system.solve(F, rtol=rtol, max_iter=max_iter, precond=_PRECOND[preconditioner],
                         precision=_PRECISION[precision], inner_rtol=inner_rtol, chunk=chunk)
    if st["status"] == -4:
        raise RuntimeError("PCG breakdown (p^T K p <= 0 or non-finite): matrix not SPD?")
    K.last_stats = st
    return u, st["iterations"], st["rel_res"], time.perf_counter() - t0


def solve_c3d10_multi(
    K: BSR3Matrix,
    F: np.ndarray,
    rtol: float = 1e-8,
    max_iter: int = 2000,
    preconditioner: str = "amg",
    precision: str = "mixed_fp32",
    amg_params=None,
    chunk: int = 8,
):
    """Several load cases at once -> (U, stats); F is (n, k), one load case per column.

    No reference counterpart: the reference runs solve_c3d10_pcg once per load case
    (solid_solver.py:197-308).  Here the cases go through the GPU in batches of 32 that share
    every matrix read, each case with its own PCG recurrence and its own stopping test on the
    FP64 true residual.  ``precision``: "fp64" or "mixed_fp32" (FP32 V-cycle in FP64 PCG).
    stats adds ``case_iterations`` and ``case_rel_res`` (arrays of k).
    """
    if preconditioner not in _PRECOND:
        raise ValueError(f"preconditioner must be one of {sorted(_PRECOND)}, got {preconditioner!r}")
    if precision not in ("fp64", "mixed_fp32"):
        raise ValueError(f"precision must be 'fp64' or 'mixed_fp32' for several load cases, got {precision!r}")
    system = K.system
    if preconditioner == "amg" and (amg_params is not None or not system.amg_ready):
        system.amg_setup(amg_params)
    U, st = system.solve_multi(F, rtol=rtol, max_iter=max_iter, precond=_PRECOND[preconditioner],
                               precision=_PRECISION[precision], chunk=chunk)
    if st["status"] == -4:
        raise RuntimeError("PCG breakdown (p^T K p <= 0 or non-finite): matrix not SPD?")
    K.last_stats = st
    return U, st


def solve_c3d10_system(
    K: BSR3Matrix,
    F: np.ndarray,
    method: str = "auto",
    rtol: float = 1e-6,
    max_iter: int = 2000,
    preconditioner: str = "jacobi",
    precision: str = "fp64",
):
    """Unified solve -> (u, stats) (solid_solver.py:132-194); defaults are the reference's.

    ``method``: "pcg" (GPU PCG), "auto" (the same: the GPU path has no size threshold), or
    "direct" -- the reference's SuperLU branch (:164-183) has no GPU counterpart here and
    raises.  Stats keep the reference's keys (method, iterations, solve_time_sec, rel_res)
    and add outer_iters, dof_per_s, setup_time_sec and levels.
    """
    if method == "direct":
        raise NotImplementedError("direct sparse factorisation is not part of the GPU path; use method='pcg'")
    if method not in ("auto", "pcg"):
        raise ValueError(f"method must be 'auto', 'pcg' or 'direct', got {method!r}")
    u, iters, rel, secs = solve_c3d10_pcg(K, F, rtol=rtol, max_iter=max_iter, preconditioner=preconditioner,
                                          precision=precision)
    st = K.last_stats
    stats = {
        "method": f"pcg_{preconditioner}_{precision}",
        "iterations": iters,
        "solve_time_sec": secs,
        "rel_res": rel,
        "outer_iters": st["outer_iterations"],
        "device_solve_sec": st["solve_seconds"],
        "setup_time_sec": st["setup_seconds"],
        "levels": st["n_levels"],
        "status": st["status"],
        "dof_per_s": K.shape[0] / st["solve_seconds"] if st["solve_seconds"] > 0 else float("inf"),
        "algorithmic_bytes": st["algorithmic_bytes"],
        "achieved_GBps": st["algorithmic_bytes"] / st["solve_seconds"] / 1e9 if st["solve_seconds"] > 0 else 0.0,
    }
    return u, stats


def compute_c3d10_stress_field(model: FEAModel, u_3dof: np.ndarray):
    """Cell stresses (M, 6), cell von Mises (M,), nodal von Mises (N,) on the GPU."""
    system = solid_system(model)
    props = solid_element_props(model)
    if system.props is None or not np.array_equal(system.props, props):
        # stresses need the element moduli on the device; assemble once if not done yet
        system.assemble(props, apply_bcs=system.bcs_applied)
    return system.stress_field(np.asarray(u_3dof, dtype=np.float64))
