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


def compute_c3d10_stress_field(model: FEAModel, u_3dof: np.ndarray):
    """Cell stresses (M, 6), cell von Mises (M,), nodal von Mises (N,) on the GPU."""
    system = solid_system(model)
    props = solid_element_props(model)
    if system.props is None or not np.array_equal(system.props, props):
        # stresses need the element moduli on the device; assemble once if not done yet
        system.assemble(props, apply_bcs=system.bcs_applied)
    return system.stress_field(np.asarray(u_3dof, dtype=np.float64))
