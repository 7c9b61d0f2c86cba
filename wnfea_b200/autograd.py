"""Differentiable compliance of a C3D10 model: ``torch.autograd.Function`` over the GPU path.

No reference counterpart (the reference has no adjoint and no autograd).  For
K(E) u = F with the Dirichlet rows of the model, the compliance C = F^T u is self-adjoint:

    dC/dE_e = -u_e^T (dK/dE_e) u_e = -u_e^T Ke u_e / E_e,      dC/dF = 2 u  (0 on fixed DOFs),

so the backward pass reuses the forward displacement and one element kernel
(``wn_adjoint_compliance_device``: Ke u_e recomputed matrix-free, dotted with u_e) -- no
second solve.  Forward: GPU assembly with the per-element moduli, AMG-PCG solve (mixed or
FP64), C = F^T u.  PyTorch only carries device memory, the stream and the autograd graph.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .amg import AMGParams
from .system import SolidSystem

_PRECISION = {"fp64": 0, "mixed_fp32": 1, "mixed_fp32_ir": 2}


class ComplianceProblem:
    """A C3D10 mesh with fixed DOFs and a Poisson ratio, solved on the GPU for any E and F.

    ``reuse_hierarchy``: build the AMG hierarchy once (at the first forward) and keep it for
    later moduli.  The solve still uses the current K in its Krylov SpMV and stops on the
    true residual of the current K, so results are exact; only the preconditioner's quality
    depends on how far E has moved (re-build with ``rebuild_hierarchy()``).
    """

    def __init__(self, nodes, conn, fixed_dofs, nu=0.3, precision="mixed_fp32", rtol=1e-8,
                 max_iter=5000, reuse_hierarchy=True, amg_params: AMGParams | None = None):
        if precision not in _PRECISION:
            raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
        self.system = SolidSystem(nodes, conn)
        self.system.set_fixed(fixed_dofs)
        self.n_el = self.system.n_el
        self.n_dof = 3 * self.system.n_nodes
        self.nu = float(nu)
        self.precision = precision
        self.rtol = rtol
        self.max_iter = max_iter
        self.reuse = reuse_hierarchy
        self.amg_params = amg_params
        self._have_hierarchy = False
        self.fixed_mask = torch.from_numpy(self.system.fixed_mask.astype(bool)).cuda()
        self.last_stats = None

    @classmethod
    def from_model(cls, model, **kw):
        from .model import solid_element_props, solid_fixed_dofs

        props = solid_element_props(model)
        return cls(model.mesh_nodes, model.solid_elements, solid_fixed_dofs(model), nu=float(props[0, 1]), **kw)

    def rebuild_hierarchy(self):
        self._have_hierarchy = False

    # -- the two GPU halves ----------------------------------------------------------------
    def solve(self, E: torch.Tensor, F: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """u with K(E) u = F (fixed DOFs of F zeroed); returns (u, F_bc)."""
        E = E.detach().to(device="cuda", dtype=torch.float64).contiguous()
        if E.shape != (self.n_el,):
            raise ValueError(f"E must have shape ({self.n_el},)")
        Fb = F.detach().to(device="cuda", dtype=torch.float64).clone()
        Fb[self.fixed_mask] = 0.0
        props = torch.stack([E, torch.full_like(E, self.nu)], dim=1).contiguous()
        stream = torch.cuda.current_stream().cuda_stream
        h = self.system.handle
        _lib.call("wn_assemble_c3d10_device", h, props.data_ptr(), 1, stream)
        self.system.props = None  # device props now differ from any host copy
        self.system.bcs_applied = True
        if not (self.reuse and self._have_hierarchy):
            prm = (self.amg_params or AMGParams()).to_c()
            _lib.call("wn_amg_setup", h, C.byref(prm))
            self._have_hierarchy = True
        u = torch.empty_like(Fb)
        sp = _lib.SolveParams(self.rtol, self.max_iter, 2, _PRECISION[self.precision], 0.0, 10, 8, 1)
        st = _lib.SolveStats()
        _lib.call("wn_solve_device", h, Fb.data_ptr(), u.data_ptr(), C.byref(sp), C.byref(st), stream)
        self.last_stats = {f: getattr(st, f) for f, _ in _lib.SolveStats._fields_}
        if st.status != 0:
            raise RuntimeError(f"compliance solve did not converge: status {st.status}, rel_res {st.rel_res:.3e}")
        return u, Fb

    def gradient(self, u: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """(dC/dE, dC/dF) at the solution u of the last assembled moduli."""
        gE = torch.empty(self.n_el, dtype=torch.float64, device="cuda")
        gF = torch.empty(self.n_dof, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        _lib.call("wn_adjoint_compliance_device", self.system.handle, u.data_ptr(), gE.data_ptr(), gF.data_ptr(),
                  stream)
        return gE, gF

    def energy_compliance(self, u: torch.Tensor, Fb: torch.Tensor) -> float:
        """2 F^T u - u^T K u: equals F^T u at the exact solution, with an error quadratic in
        the solve error (used for finite-difference checks)."""
        Ku = torch.empty_like(u)
        stream = torch.cuda.current_stream().cuda_stream
        _lib.call("wn_spmv_solid_device", self.system.handle, 0, u.data_ptr(), Ku.data_ptr(), stream)
        return float(2.0 * torch.dot(Fb, u) - torch.dot(u, Ku))

    def compliance(self, E: torch.Tensor, F: torch.Tensor) -> torch.Tensor:
        return Compliance.apply(E, F, self)


class Compliance(torch.autograd.Function):
    """C(E, F) = F^T u with K(E) u = F; backward by the self-adjoint formula."""

    @staticmethod
    def forward(ctx, E, F, problem: ComplianceProblem):
        u, Fb = problem.solve(E, F)
        ctx.problem = problem
        ctx.save_for_backward(u)
        return torch.dot(Fb, u).reshape(())

    @staticmethod
    def backward(ctx, grad_c):
        (u,) = ctx.saved_tensors
        gE, gF = ctx.problem.gradient(u)
        return grad_c * gE, grad_c * gF, None


def compliance(E: torch.Tensor, F: torch.Tensor, problem: ComplianceProblem) -> torch.Tensor:
    """Functional form of ``Compliance.apply``."""
    return Compliance.apply(E, F, problem)
