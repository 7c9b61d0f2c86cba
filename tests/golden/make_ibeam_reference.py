"""Run the REFERENCE's own C3D10 CPU solve to convergence on the full 200,340-element I-beam and
record what it did, as the fixture ``ibeam_reference_jacobi.json`` of this directory.

    python tests/golden/make_ibeam_reference.py /path/to/reference

The reference (wnfea) is imported read-only with ``builtins.Path`` set first (wnfea/model.py:191
annotates with ``Path`` without importing it).  The mesh comes from this repository's structured
I-beam generator (315 slices, seed 0: 200,340 elements, 1,012,755 DOFs) and is handed, as
arrays, to the reference's own functions:

* ``assemble_c3d10_sparse_3dof(model)``            (wnfea/solver/solid_solver.py:26-129)
* ``solve_c3d10_pcg(K, F, rtol=1e-8, max_iter=200000, preconditioner="jacobi")``
                                                    (wnfea/solver/solid_solver.py:197-308)

scipy's ``cg`` with the point-Jacobi preconditioner runs single-threaded, about 85 ms per
iteration on one host core, so the solve takes about an hour.  The fixture keeps the iteration
count, the wall times, the final relative residual and a strided sample of the displacement;
``bench.py --impl reference`` uses the iteration count of this run to turn its timed sample of
iterations into a solve time, and the GPU tests compare the sample with the GPU solution.
"""

from __future__ import annotations

import builtins
import json
import os
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
SAMPLE_STRIDE = 97


def main(ref: str) -> None:
    builtins.Path = pathlib.Path
    sys.path.insert(0, ref)
    sys.path.insert(0, str(ROOT))
    import scipy
    import wnfea
    from wnfea.solver.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_pcg

    from wnfea_b200.mesh import generate_c3d10_ibeam_structured

    m, meta = generate_c3d10_ibeam_structured(n_slices=315, length=4.0, seed=0)
    rm = wnfea.FEAModel()
    rm.mesh_nodes = m.mesh_nodes
    rm.solid_elements = m.solid_elements
    for name, mat in m.materials.items():
        rm.materials[name] = wnfea.MaterialDef(name, mat.youngs_modulus, mat.poissons_ratio, mat.yield_strength)
    rm.solid_materials = {i: next(iter(m.materials)) for i in range(len(m.solid_elements))}
    for s in m.supports:
        rm.supports.append(wnfea.create_fixed_support(s.node_id, is_geometry_node=False))
    for ld in m.loads:
        rm.loads.append(wnfea.LoadDef(node_id=ld.node_id, is_geometry_node=False, fx=ld.fx, fy=ld.fy, fz=ld.fz))

    t0 = time.perf_counter()
    K, F, fixed = assemble_c3d10_sparse_3dof(rm)
    t_asm = time.perf_counter() - t0
    print(f"assembly {t_asm:.1f} s, n {K.shape[0]}, nnz {K.nnz}", flush=True)
    t0 = time.perf_counter()
    u, iters, rel, t_solve = solve_c3d10_pcg(K, F, rtol=1e-8, max_iter=200000, preconditioner="jacobi")
    wall = time.perf_counter() - t0
    true_rel = float(np.linalg.norm(F - K @ u) / np.linalg.norm(F))
    out = {
        "workload": f"C3D10 I-beam {meta['n_elements']} el / {K.shape[0]} DOFs (315 slices, seed 0)",
        "reference_calls": ["assemble_c3d10_sparse_3dof(model)",
                            "solve_c3d10_pcg(K, F, rtol=1e-8, max_iter=200000, preconditioner='jacobi')"],
        "n_dofs": int(K.shape[0]),
        "nnz": int(K.nnz),
        "assembly_s": t_asm,
        "iterations": int(iters),
        "solve_s": float(t_solve),
        "solve_wall_s": wall,
        "s_per_iteration": float(t_solve) / max(int(iters), 1),
        "final_rel_res": float(rel),
        "true_rel_res": true_rel,
        "cores": 1,
        "threads_env": {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS")},
        "numpy": np.__version__,
        "scipy": scipy.__version__,
        "u_sample_stride": SAMPLE_STRIDE,
        "u_sample": [float(v) for v in u[::SAMPLE_STRIDE]],
        "u_tip_min_z": float(u.reshape(-1, 3)[:, 2].min()),
    }
    (HERE / "ibeam_reference_jacobi.json").write_text(json.dumps(out, indent=1))
    print(json.dumps({k: v for k, v in out.items() if k != "u_sample"}), flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
