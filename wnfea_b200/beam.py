"""Co-rotational 3D beam path with the reference's API, evaluated on the GPU.

* ``prepare_batch_data(model)``        -- element arrays as fast_kernels.py:263-306 packs them
                                          (props [E, G, A, Iy, Iz, J], reference triads, L0);
* ``compute_internal_forces_fast(model, U_full, F_int=None, device="gpu")``
                                       -- fast_kernels.py:359-537: beams and C3D10 solids at
                                          6 DOFs per node, both through libwnfea_cuda;
* ``BeamFrame``                        -- GPU handle: internal force, consistent tangent
                                          (6x6-block BSR), block-Jacobi BiCGStab;
* ``solve_nonlinear_jfnk(model, ...)`` -- nonlinear_solver.py:159-376: incremental load
                                          steps, Newton with Eisenstat-Walker forcing and
                                          Armijo backtracking.  The Newton system uses the
                                          exact consistent tangent assembled on the GPU
                                          instead of finite-difference Jacobian-vector
                                          products (jfnk_operator.py:98-134); the residual
                                          and its Dirichlet rows follow residual.py:125-166.
"""

from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import call, ptr
from .model import DOFType, FEAModel, solid_element_props


class NonLinearConvergenceError(Exception):
    """Newton did not converge within max_newton_iter (nonlinear_solver.py:46)."""


@dataclass
class BatchModelData:
    nodes: np.ndarray
    beam_elements: np.ndarray
    beam_props: np.ndarray
    beam_e_ref: np.ndarray
    beam_L0: np.ndarray
    n_beams: int
    n_nodes: int


def prepare_batch_data(model: FEAModel) -> BatchModelData:
    """Contiguous beam arrays (fast_kernels.py:263-306): the reference triad takes
    e2 = ref x e1 with ref = z unless |e1_z| >= 0.9 (then y), e3 = e1 x e2."""
    nodes = np.ascontiguousarray(model.mesh_nodes, dtype=np.float64)
    if model.mesh_elements is None or len(model.mesh_elements) == 0:
        z = np.empty((0,))
        return BatchModelData(nodes, np.empty((0, 2), np.int32), z.reshape(0, 6), z.reshape(0, 9), z, 0, len(nodes))
    el = np.ascontiguousarray(model.mesh_elements, dtype=np.int32)
    props = np.zeros((len(el), 6))
    for e in range(len(el)):
        a = model.element_properties[e]
        m = model.materials[a.material_name]
        s = model.sections[a.section_name]
        props[e] = [m.youngs_modulus, m.shear_modulus, s.area, s.iy, s.iz, s.j]
    v0 = nodes[el[:, 1]] - nodes[el[:, 0]]
    L0 = np.linalg.norm(v0, axis=1)
    e1 = v0 / np.maximum(L0[:, None], 1e-15)
    ref = np.where((np.abs(e1[:, 2]) < 0.9)[:, None], [0.0, 0.0, 1.0], [0.0, 1.0, 0.0])
    e2 = np.cross(ref, e1)
    e2 /= np.linalg.norm(e2, axis=1, keepdims=True)
    e3 = np.cross(e1, e2)
    e3 /= np.linalg.norm(e3, axis=1, keepdims=True)
    eref = np.ascontiguousarray(np.hstack([e1, e2, e3]))
    return BatchModelData(nodes, el, np.ascontiguousarray(props), eref, np.ascontiguousarray(L0), len(el), len(nodes))


def compute_internal_forces_fast(model: FEAModel, U_full: np.ndarray, F_int: np.ndarray | None = None,
                                 device: str = "gpu", block_size: int = 0, grid_size: int = 0) -> np.ndarray:
    """Global internal force (n_nodes * 6,) of beams and C3D10 solids (fast_kernels.py:359-537).

    ``device`` is accepted for signature compatibility; every evaluation runs on the GPU.
    ``block_size`` / ``grid_size`` are ignored (launch shapes are chosen by the library).
    """
    b = getattr(model, "_wn_batch", None)
    if b is None or b.n_nodes != len(model.mesh_nodes):
        b = prepare_batch_data(model)
        object.__setattr__(model, "_wn_batch", b)
    U = np.ascontiguousarray(U_full, dtype=np.float64)
    if F_int is None:
        F_int = np.zeros(b.n_nodes * 6)
    else:
        F_int.fill(0.0)
    if b.n_beams:
        call("wn_beam_internal_forces", ptr(b.nodes), ptr(b.beam_elements), ptr(b.beam_props), ptr(b.beam_e_ref),
             ptr(b.beam_L0), ptr(U), ptr(F_int), b.n_beams, b.n_nodes)
    if model.solid_elements is not None and len(model.solid_elements):
        conn = np.ascontiguousarray(model.solid_elements, dtype=np.int32)
        props = np.ascontiguousarray(solid_element_props(model))
        call("wn_c3d10_internal_forces", ptr(b.nodes), ptr(conn), ptr(props), ptr(U), ptr(F_int), len(conn),
             b.n_nodes)
    return F_int


class BeamFrame:
    """GPU handle of a beam frame: f_int, consistent tangent (BSR6), BiCGStab."""

    def __init__(self, model: FEAModel):
        self.data = prepare_batch_data(model)
        d = self.data
        h = C.c_void_p()
        call("wn_beam_create", d.n_nodes, d.n_beams, ptr(d.nodes), ptr(d.beam_elements), ptr(d.beam_props),
             ptr(d.beam_e_ref), ptr(d.beam_L0), C.byref(h))
        self._h = h
        self.n = 6 * d.n_nodes

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().wn_beam_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fixed(self, mask: np.ndarray | None):
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        call("wn_beam_set_fixed", self._h, ptr(m))

    def internal_force(self, U: np.ndarray) -> np.ndarray:
        f = np.empty(self.n)
        call("wn_beam_evaluate", self._h, ptr(np.ascontiguousarray(U, dtype=np.float64)), ptr(f), 0, 0)
        return f

    def assemble_tangent(self, U: np.ndarray, apply_bcs: bool = True, with_force: bool = False):
        f = np.empty(self.n) if with_force else None
        call("wn_beam_evaluate", self._h, ptr(np.ascontiguousarray(U, dtype=np.float64)), ptr(f), 1, int(apply_bcs))
        return f

    def tangent_bsr(self):
        import scipy.sparse as sp

        nn, ne, nb = C.c_int64(), C.c_int64(), C.c_int64()
        call("wn_beam_info", self._h, C.byref(nn), C.byref(ne), C.byref(nb))
        rp = np.empty(nn.value + 1, dtype=np.int32)
        ci = np.empty(nb.value, dtype=np.int32)
        call("wn_beam_get_pattern", self._h, ptr(rp), ptr(ci))
        v = np.empty((nb.value, 6, 6))
        call("wn_beam_get_tangent", self._h, ptr(v))
        return sp.bsr_matrix((v, ci, rp), shape=(self.n, self.n))

    def solve(self, rhs: np.ndarray, rtol: float = 1e-10, max_iter: int = 2000, method: str = "auto"):
        """x with K_t x = rhs: "dense" (LU on the GPU, small frames), "bicgstab" (6x6 block
        Jacobi) or "auto"; returns (x, iterations, rel_res, status)."""
        x = np.empty(self.n)
        it, rr = C.c_int(), C.c_double()
        code = {"auto": 0, "dense": 1, "bicgstab": 2}[method]
        rc = _lib.lib().wn_beam_solve(self._h, ptr(np.ascontiguousarray(rhs, dtype=np.float64)), ptr(x), code, rtol,
                                      max_iter, C.byref(it), C.byref(rr))
        if rc not in (0, -5, -4):
            raise _lib.WnError("wn_beam_solve", rc, _lib.last_error())
        return x, it.value, rr.value, rc


class FrameSystem:
    """A linear 6-DOF-per-node system on the GPU (``wn_beam_linear_system``): smoothed-
    aggregation AMG over the 6 rigid-body modes of beam nodes and PCG, in FP64 or with an FP32
    V-cycle -- the B200 counterpart of BlockBeamAMGPreconditioner.solve_pcg ->
    hip_solve_pcg_amg (fast_kernels.py:598-663)."""

    def __init__(self, frame: BeamFrame):
        h = C.c_void_p()
        call("wn_beam_linear_system", frame._h, C.byref(h))
        self._h = h
        self.n = frame.n

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().wn_solid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def amg_setup(self, params=None) -> float:
        from .amg import AMGParams

        prm = (params or AMGParams()).to_c()
        t0 = time.perf_counter()
        call("wn_amg_setup", self._h, C.byref(prm))
        return time.perf_counter() - t0

    def solve(self, F: np.ndarray, rtol: float = 1e-8, max_iter: int = 2000, precision: str = "mixed_fp32",
              chunk: int = 8):
        """U with K U = F (F zero on fixed DOFs); returns (U, stats dict)."""
        prec = {"fp64": 0, "mixed_fp32": 1}[precision]
        F = np.ascontiguousarray(F, dtype=np.float64)
        U = np.empty_like(F)
        prm = _lib.SolveParams(rtol, max_iter, 2, prec, 0.0, 10, chunk, 1)
        st = _lib.SolveStats()
        call("wn_solve", self._h, ptr(F), ptr(U), C.byref(prm), C.byref(st))
        return U, {f: getattr(st, f) for f, _ in _lib.SolveStats._fields_}

    def solve_device(self, F, U, rtol: float = 1e-8, max_iter: int = 2000, precision: str = "mixed_fp32",
                     stream: int = 0):
        prm = _lib.SolveParams(rtol, max_iter, 2, {"fp64": 0, "mixed_fp32": 1}[precision], 0.0, 10, 8, 1)
        st = _lib.SolveStats()
        call("wn_solve_device", self._h, _lib.dptr(F), _lib.dptr(U), C.byref(prm), C.byref(st), stream)
        return {f: getattr(st, f) for f, _ in _lib.SolveStats._fields_}


def frame_linear_system(model: FEAModel) -> tuple[BeamFrame, FrameSystem, np.ndarray]:
    """(frame, system, F): the frame's stiffness at U = 0 with its fixed DOFs made identity,
    as a GPU AMG-PCG system, and the load vector with zeros on the fixed DOFs.  Only fixed
    (zero) supports: a prescribed non-zero value raises."""
    dofs, vals = get_boundary_constraints(model)
    if np.any(vals != 0.0):
        raise ValueError("frame_linear_system: prescribed non-zero displacements are not supported")
    frame = BeamFrame(model)
    mask = np.zeros(frame.n, dtype=np.uint8)
    mask[dofs] = 1
    frame.set_fixed(mask)
    frame.assemble_tangent(np.zeros(frame.n), apply_bcs=True)
    F = build_external_force_vector(model)
    F[dofs] = 0.0
    return frame, FrameSystem(frame), F


def solve_frame_linear(model: FEAModel, rtol: float = 1e-8, precision: str = "mixed_fp32", amg_params=None,
                       max_iter: int = 2000):
    """Linear static solve of a beam frame on the GPU -> (U (n_nodes * 6,), stats)."""
    frame, system, F = frame_linear_system(model)
    setup_s = system.amg_setup(amg_params)
    U, st = system.solve(F, rtol=rtol, max_iter=max_iter, precision=precision)
    st["setup_seconds"] = setup_s
    system.close()
    frame.close()
    return U, st


def _mesh_node(model: FEAModel, node_id: int, is_geometry_node: bool):
    if is_geometry_node:
        return model.geometry_to_mesh_node_map.get(node_id)
    return node_id


def build_external_force_vector(model: FEAModel) -> np.ndarray:
    """Unscaled nodal loads (n_nodes * 6,) (residual.py:20-47)."""
    n = len(model.mesh_nodes)
    F = np.zeros(n * 6)
    for ld in model.loads:
        nid = _mesh_node(model, ld.node_id, ld.is_geometry_node)
        if nid is None or nid >= n:
            continue
        F[nid * 6 : nid * 6 + 6] += ld.force_vector
    return F


def get_boundary_constraints(model: FEAModel) -> tuple[np.ndarray, np.ndarray]:
    """Constrained DOFs and prescribed values (residual.py:50-92)."""
    n = len(model.mesh_nodes)
    dofs, vals = [], []
    for s in model.supports:
        nid = _mesh_node(model, s.node_id, s.is_geometry_node)
        if nid is None or nid >= n:
            continue
        for k, c in enumerate(s.constraints):
            if c.dof_type == DOFType.FIXED:
                dofs.append(nid * 6 + k)
                vals.append(0.0)
            elif c.dof_type == DOFType.PRESCRIBED:
                dofs.append(nid * 6 + k)
                vals.append(float(c.value))
    return np.asarray(dofs, dtype=np.int64), np.asarray(vals)


def solve_nonlinear_jfnk(model: FEAModel, n_load_steps: int = 5, max_newton_iter: int = 25, tol_rel: float = 1e-5,
                         tol_abs: float = 1e-5, use_amg: bool = True, use_mixed_precision: bool = False,
                         use_tri_precision: bool = False, switch_tol: float = 1e-2, verbose: bool = True,
                         stats: dict | None = None) -> np.ndarray:
    """Geometrically nonlinear beam-frame solve (nonlinear_solver.py:159-376 signature).

    Load factors lambda = k / n_load_steps; per step Newton on R(U) = F_int(U) - lambda F_ext
    with R_c = U_c - lambda u_c on constrained DOFs; the Newton system K_t(U) dU = -R uses the
    GPU consistent tangent (constrained rows/columns identity) solved by BiCGStab to the
    Eisenstat-Walker tolerance min(0.1, 0.5 (|R|/|R_prev|)^2) (floor 1e-10 absolute, as
    :289-292); Armijo backtracking halves the step while |R| does not decrease, down to
    1/16 (:312-335).  ``use_amg`` / precision flags are accepted for compatibility (the
    frame's linear systems are solved in FP64).  Returns U (n_nodes * 6,) and sets
    ``model.displacements``.
    """
    errors = model.validate_for_solving()
    if errors:
        raise ValueError("Cannot solve model:\n  " + "\n  ".join(errors))
    if model.solid_elements is not None and len(model.solid_elements):
        raise NotImplementedError("mixed beam-solid models are not on this path")
    frame = BeamFrame(model)
    n = frame.n
    F_ext = build_external_force_vector(model)
    cdofs, cvals = get_boundary_constraints(model)
    mask = np.zeros(n, dtype=np.uint8)
    mask[cdofs] = 1
    frame.set_fixed(mask)
    U = np.zeros(n)
    t0 = time.perf_counter()
    total_lin = 0
    newton_total = 0

    def residual(Uv, lam):
        R = frame.internal_force(Uv) - lam * F_ext
        if len(cdofs):
            R[cdofs] = Uv[cdofs] - lam * cvals
        return R

    for step, lam in enumerate(np.linspace(1.0 / n_load_steps, 1.0, n_load_steps), 1):
        R = residual(U, lam)
        r0 = float(np.linalg.norm(R))
        prev = r0
        if r0 < tol_abs:
            continue
        for it in range(1, max_newton_iter + 1):
            rn = float(np.linalg.norm(R))
            if rn < tol_abs or rn / (r0 + 1e-20) < tol_rel:
                break
            eta = min(0.1, 0.5 * (rn / (prev + 1e-20)) ** 2)
            inner = max(eta * rn, 1e-10) / (rn + 1e-20)
            frame.assemble_tangent(U, apply_bcs=True)
            dU, lin_its, lin_rel, status = frame.solve(-R, rtol=max(inner, 1e-14), max_iter=4 * n)
            total_lin += lin_its
            newton_total += 1
            prev = rn
            alpha = 1.0
            Ut = U + alpha * dU
            Rt = residual(Ut, lam)
            tn = float(np.linalg.norm(Rt))
            while tn >= rn and alpha > 0.0625:
                alpha *= 0.5
                Ut = U + alpha * dU
                Rt = residual(Ut, lam)
                tn = float(np.linalg.norm(Rt))
            U, R = Ut, Rt
            if verbose:
                print(f"  step {step} Newton {it:2d}: |R| = {tn:.4e} (rel {tn / (r0 + 1e-20):.2e}) "
                      f"BiCGStab {lin_its} step {alpha:.3f}")
        else:
            raise NonLinearConvergenceError(
                f"Newton failed to converge at load step {step} (lambda={lam:.3f}); |R| = {np.linalg.norm(R):.4e}")
    if stats is not None:
        stats.update({"newton_iterations": newton_total, "linear_iterations": total_lin,
                      "solve_time_sec": time.perf_counter() - t0})
    model.displacements = U
    return U
