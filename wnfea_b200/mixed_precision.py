"""Precision configuration (wnfea/solver/mixed_precision.py:23-122).

``PrecisionConfig``, the presets and the cast helpers keep the reference's fields and names.
On this path a configuration selects the solver's ``precision`` argument
(``solver_precision``):

* ``enabled`` with ``inner_dtype = float32`` -> ``"mixed_fp32"``: FP64 PCG (FP64 SpMV, x, r, q
  and dot products; FP32 search directions on the streamed fine level) preconditioned in FP32 (the AMG V-cycle with FP32 values, vectors and
  accumulation and an FP64 coarsest inverse), inside the FP64 true-residual loop;
* otherwise (``FULL_FP64``) -> ``"fp64"``.

* ``use_tri_precision`` (``TRI_PRECISION``) -> ``"mixed_fp16"``: as ``"mixed_fp32"`` with the
  V-cycle's fine level on the diagonally equilibrated matrix stored in FP16.  The reference
  runs its FP16 V-cycles only while the relative residual is above ``switch_tol`` and FP32 ones
  after; here the equilibrated FP16 fine level is used on every iteration (the AMG-PCG
  iteration count stays within a few percent of the FP32 V-cycle's), so ``switch_tol`` is
  kept for the interface but not consulted.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class PrecisionConfig:
    inner_dtype: type = np.float32
    outer_dtype: type = np.float64
    precond_coarse_dtype: type = np.float16
    switch_tol: float = 1e-2
    use_tri_precision: bool = False
    enabled: bool = True

    @property
    def inner_eps_scale(self) -> float:
        """sqrt(eps) of the inner dtype (mixed_precision.py:66-69)."""
        return float(np.sqrt(np.finfo(self.inner_dtype).eps))

    @property
    def outer_eps_scale(self) -> float:
        """sqrt(eps) of the outer dtype (mixed_precision.py:71-74)."""
        return float(np.sqrt(np.finfo(self.outer_dtype).eps))

    @property
    def working_dtype(self):
        return np.dtype(self.inner_dtype) if self.enabled else np.dtype(self.outer_dtype)

    @property
    def solver_precision(self) -> str:
        """The ``precision`` argument of solve_c3d10_pcg this configuration selects."""
        if not (self.enabled and np.dtype(self.inner_dtype) == np.float32):
            return "fp64"
        return "mixed_fp16" if self.use_tri_precision else "mixed_fp32"

    def summary(self) -> str:
        if not self.enabled:
            return f"Uniform {np.dtype(self.outer_dtype).name} (mixed precision disabled)"
        inner = np.dtype(self.inner_dtype).name
        outer = np.dtype(self.outer_dtype).name
        if self.use_tri_precision:
            return (f"Tri-precision: {outer} PCG/residual/dots, {inner} AMG V-cycle with its fine level in "
                    f"float16 (equilibrated)")
        return f"Mixed precision: {outer} PCG/residual/dots, {inner} preconditioner (AMG V-cycle)"


MIXED_FP32 = PrecisionConfig(inner_dtype=np.float32, outer_dtype=np.float64, enabled=True, use_tri_precision=False)
TRI_PRECISION = PrecisionConfig(inner_dtype=np.float32, outer_dtype=np.float64, precond_coarse_dtype=np.float16,
                                switch_tol=1e-2, use_tri_precision=True, enabled=True)
FULL_FP64 = PrecisionConfig(inner_dtype=np.float64, outer_dtype=np.float64, enabled=False, use_tri_precision=False)


def cast_to_inner(arr: np.ndarray, config: PrecisionConfig) -> np.ndarray:
    """``arr`` in the configuration's working dtype (mixed_precision.py:109-114)."""
    target = config.working_dtype
    return arr if arr.dtype == target else arr.astype(target, copy=False)


def cast_to_outer(arr: np.ndarray, config: PrecisionConfig) -> np.ndarray:
    """``arr`` in the outer (accumulation) dtype (mixed_precision.py:117-122)."""
    target = np.dtype(config.outer_dtype)
    return arr if arr.dtype == target else arr.astype(target, copy=False)
