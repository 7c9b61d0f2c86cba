"""wnfea_b200 -- B200-native (sm_100a) implementation of WNFEA's linear-elastic solve path.

The public names follow the reference package ``wnfea`` (wnfea/__init__.py) for the C3D10
solid and co-rotational beam path; every numerical kernel runs on the GPU through the C ABI
of ``libwnfea_cuda.so`` (include/wnfea_cuda.h).
"""

from .model import (
    DOFConstraint,
    DOFType,
    FEAModel,
    LoadDef,
    MaterialDef,
    PropertyAssignment,
    SectionDef,
    SupportDef,
    create_fixed_support,
    create_rectangular_bar,
)
from .autograd import Compliance, ComplianceProblem
from .beam import (
    BeamFrame,
    NonLinearConvergenceError,
    compute_internal_forces_fast,
    prepare_batch_data,
    solve_nonlinear_jfnk,
)
from .rcm import (
    apply_rcm_to_model,
    compute_matrix_bandwidth,
    compute_node_adjacency_matrix,
    compute_rcm_order,
    permute_solution_to_original,
)
from .vtu import VTUExporter, export_vtu
from .mesh import generate_c3d10_structured_block
from .elements import element_internal_forces_c3d10, element_stiffness_c3d10, element_stresses_c3d10
from .mixed_precision import FULL_FP64, MIXED_FP32, TRI_PRECISION, PrecisionConfig
from .solid_solver import (
    assemble_c3d10_sparse_3dof,
    compute_c3d10_stress_field,
    solve_c3d10_multi,
    solve_c3d10_pcg,
    solve_c3d10_system,
)

__all__ = [
    "FEAModel", "MaterialDef", "SectionDef", "PropertyAssignment",
    "SupportDef", "LoadDef", "DOFConstraint", "DOFType", "create_fixed_support", "create_rectangular_bar",
    "assemble_c3d10_sparse_3dof", "compute_c3d10_stress_field", "solve_c3d10_pcg", "solve_c3d10_system",
    "solve_c3d10_multi",
    "PrecisionConfig", "MIXED_FP32", "FULL_FP64", "TRI_PRECISION",
    "compute_internal_forces_fast", "prepare_batch_data", "solve_nonlinear_jfnk", "NonLinearConvergenceError",
    "BeamFrame", "ComplianceProblem", "Compliance",
    "apply_rcm_to_model", "compute_matrix_bandwidth", "compute_node_adjacency_matrix", "compute_rcm_order",
    "permute_solution_to_original", "VTUExporter", "export_vtu", "generate_c3d10_structured_block",
    "element_stiffness_c3d10", "element_internal_forces_c3d10", "element_stresses_c3d10",
]
