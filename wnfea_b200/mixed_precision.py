"""Precision configuration (wnfea/solver/mixed_precision.py:23-106).

``PrecisionConfig`` and the presets keep the reference's fields.  On this path they select
the solver precision: ``enabled`` with ``inner_dtype = float32`` means FP32 inner PCG + AMG
(FP32 values, FP32 accumulation, FP64 dot products) inside FP64 iterative refinement
(``precision="mixed_fp32"``); ``FULL_FP64`` is the plain FP64 path.  The FP16
``TRI_PRECISION`` preset is accepted and runs as ``MIXED_FP32`` (no FP16 V-cycle here).
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
    def working_dtype(self):
        return np.dtype(self.inner_dtype) if self.enabled else np.dtype(self.outer_dtype)

    @property
    def solver_precision(self) -> str:
        """The ``precision`` argument of solve_c3d10_pcg this configuration selects."""
        return "mixed_fp32" if self.enabled and np.dtype(self.inner_dtype) == np.float32 else "fp64"

    def summary(self) -> str:
        if not self.enabled:
            return f"Uniform {np.dtype(self.outer_dtype).name} (mixed precision disabled)"
        return (f"Mixed precision: inner={np.dtype(self.inner_dtype).name} (PCG/AMG), "
                f"outer={np.dtype(self.outer_dtype).name} (residual/accumulation)")


MIXED_FP32 = PrecisionConfig(inner_dtype=np.float32, outer_dtype=np.float64, enabled=True, use_tri_precision=False)
TRI_PRECISION = PrecisionConfig(inner_dtype=np.float32, outer_dtype=np.float64, precond_coarse_dtype=np.float16,
                                switch_tol=1e-2, use_tri_precision=True, enabled=True)
FULL_FP64 = PrecisionConfig(inner_dtype=np.float64, outer_dtype=np.float64, enabled=False, use_tri_precision=False)
