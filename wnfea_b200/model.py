"""Model, material, section and boundary-condition types of the C3D10 / beam solve path.

These keep the field names and meanings of the reference's data model so that code
written against it drives this package unchanged:

* ``FEAModel``                    -- wnfea/model.py:44-235 (mesh, materials, supports, loads)
* ``MaterialDef``                 -- wnfea/properties/materials.py:12-48
* ``SectionDef`` / section makers -- wnfea/properties/sections.py:17-66, 221-242
* ``DOFType``/``DOFConstraint``/``SupportDef``/``LoadDef``/``create_fixed_support``
                                  -- wnfea/boundary/conditions.py:17-162

Only the parts of the reference model that feed the solve path are kept (geometry import,
edge assignments and the GUI pipeline stages are out of scope).  One addition: an optional
``solid_props`` array of per-element ``[E, nu]`` rows, used when every element carries its
own modulus (the graded-modulus block); when present it takes precedence over
``solid_materials``.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from enum import Enum

import numpy as np


# --------------------------------------------------------------------------------------
# Boundary conditions  (wnfea/boundary/conditions.py)
# --------------------------------------------------------------------------------------
class DOFType(Enum):
    """Constraint type of one degree of freedom (conditions.py:17-21)."""

    FREE = "free"
    FIXED = "fixed"
    PRESCRIBED = "prescribed"


@dataclass
class DOFConstraint:
    """One DOF's constraint (conditions.py:24-39)."""

    dof_type: DOFType = DOFType.FREE
    value: float = 0.0


@dataclass
class SupportDef:
    """Per-node support: six DOFs [Ux, Uy, Uz, Rx, Ry, Rz] (conditions.py:42-102)."""

    node_id: int
    is_geometry_node: bool = True
    ux: DOFConstraint = field(default_factory=DOFConstraint)
    uy: DOFConstraint = field(default_factory=DOFConstraint)
    uz: DOFConstraint = field(default_factory=DOFConstraint)
    rx: DOFConstraint = field(default_factory=DOFConstraint)
    ry: DOFConstraint = field(default_factory=DOFConstraint)
    rz: DOFConstraint = field(default_factory=DOFConstraint)
    label: str = ""

    @property
    def constraints(self) -> list[DOFConstraint]:
        return [self.ux, self.uy, self.uz, self.rx, self.ry, self.rz]

    @property
    def has_any_constraint(self) -> bool:
        return any(c.dof_type != DOFType.FREE for c in self.constraints)

    @property
    def fixed_dof_indices(self) -> list[int]:
        return [i for i, c in enumerate(self.constraints) if c.dof_type == DOFType.FIXED]

    @property
    def prescribed_dofs(self) -> dict[int, float]:
        return {i: c.value for i, c in enumerate(self.constraints) if c.dof_type == DOFType.PRESCRIBED}


@dataclass
class LoadDef:
    """Point load on a node (conditions.py:105-146)."""

    node_id: int
    is_geometry_node: bool = True
    fx: float = 0.0
    fy: float = 0.0
    fz: float = 0.0
    mx: float = 0.0
    my: float = 0.0
    mz: float = 0.0
    label: str = ""

    @property
    def force_vector(self) -> list[float]:
        return [self.fx, self.fy, self.fz, self.mx, self.my, self.mz]

    @property
    def has_any_load(self) -> bool:
        return any(abs(v) > 1e-12 for v in self.force_vector)


def create_fixed_support(node_id: int, is_geometry_node: bool = True, label: str = "") -> SupportDef:
    """All six DOFs fixed at zero (conditions.py:149-162)."""
    return SupportDef(
        node_id=node_id,
        is_geometry_node=is_geometry_node,
        ux=DOFConstraint(DOFType.FIXED),
        uy=DOFConstraint(DOFType.FIXED),
        uz=DOFConstraint(DOFType.FIXED),
        rx=DOFConstraint(DOFType.FIXED),
        ry=DOFConstraint(DOFType.FIXED),
        rz=DOFConstraint(DOFType.FIXED),
        label=label,
    )


# --------------------------------------------------------------------------------------
# Materials and sections  (wnfea/properties/)
# --------------------------------------------------------------------------------------
@dataclass
class MaterialDef:
    """Isotropic material (materials.py:12-48); G = E / (2 (1 + nu))."""

    name: str
    youngs_modulus: float
    poissons_ratio: float
    yield_strength: float = 2.5e8

    @property
    def shear_modulus(self) -> float:
        return self.youngs_modulus / (2.0 * (1.0 + self.poissons_ratio))


@dataclass
class SectionDef:
    """Beam cross-section (sections.py:17-66)."""

    name: str
    area: float
    iy: float
    iz: float
    j: float
    outer_radius: float | None = None
    inner_radius: float = 0.0


def create_rectangular_bar(name: str, width: float, height: float) -> SectionDef:
    """Solid rectangle; torsion constant by the same series as sections.py:221-242."""
    if width <= 0 or height <= 0:
        raise ValueError("Width and height must be positive")
    area = width * height
    iy = width * height**3 / 12.0
    iz = height * width**3 / 12.0
    a, b = max(width, height), min(width, height)
    j = a * b**3 * (1.0 / 3.0 - 0.21 * (b / a) * (1.0 - b**4 / (12.0 * a**4)))
    return SectionDef(name=name, area=area, iy=iy, iz=iz, j=j, outer_radius=width / 2.0)


@dataclass
class PropertyAssignment:
    """Material + section of a beam element (model.py:37-41)."""

    material_name: str
    section_name: str


# --------------------------------------------------------------------------------------
# The model  (wnfea/model.py:44-235)
# --------------------------------------------------------------------------------------
@dataclass
class FEAModel:
    """Single source of truth for the solve path (same field names as model.py:44-90)."""

    materials: dict[str, MaterialDef] = field(default_factory=dict)
    sections: dict[str, SectionDef] = field(default_factory=dict)
    mesh_nodes: np.ndarray | None = None  # (N, 3) float64
    mesh_elements: np.ndarray | None = None  # (E_beam, 2) beam connectivity
    element_properties: dict[int, PropertyAssignment] = field(default_factory=dict)
    solid_elements: np.ndarray | None = None  # (M, 10) C3D10 connectivity
    solid_materials: dict[int, str] = field(default_factory=dict)
    solid_props: np.ndarray | None = None  # optional (M, 2) per-element [E, nu]
    supports: list[SupportDef] = field(default_factory=list)
    loads: list[LoadDef] = field(default_factory=list)
    geometry_to_mesh_node_map: dict[int, int] = field(default_factory=dict)
    displacements: np.ndarray | None = None
    element_results: dict | None = None

    def validate_for_solving(self) -> list[str]:
        """Same checks as model.py:144-160."""
        errors = []
        if self.mesh_nodes is None or (self.mesh_elements is None and self.solid_elements is None):
            errors.append("No mesh generated. Run the mesher first.")
        if not self.supports:
            errors.append("No supports defined. Add at least one boundary condition.")
        if not self.loads:
            errors.append("No loads defined. Add at least one load.")
        if self.supports and not any(s.has_any_constraint for s in self.supports):
            errors.append("No support has any constrained DOFs.")
        if self.loads and not any(ld.has_any_load for ld in self.loads):
            errors.append("All loads are zero. Add at least one nonzero load.")
        return errors


def solid_element_props(model: FEAModel) -> np.ndarray:
    """Per-element ``[E, nu]`` rows for the C3D10 elements of ``model``.

    Material lookup follows solid_solver.py:67-79: an element's ``solid_materials`` entry
    names a material; unnamed or unknown names fall back to the first material, and to
    steel (2.1e11, 0.3) when the model has none.  A ``solid_props`` array overrides this.
    """
    n_el = 0 if model.solid_elements is None else len(model.solid_elements)
    if model.solid_props is not None:
        props = np.ascontiguousarray(model.solid_props, dtype=np.float64)
        if props.shape != (n_el, 2):
            raise ValueError(f"solid_props must have shape ({n_el}, 2), got {props.shape}")
        return props
    default = next(iter(model.materials.values())) if model.materials else None
    e_def = default.youngs_modulus if default else 2.1e11
    nu_def = default.poissons_ratio if default else 0.3
    props = np.empty((n_el, 2), dtype=np.float64)
    props[:, 0] = e_def
    props[:, 1] = nu_def
    if model.solid_materials:
        for eid, name in model.solid_materials.items():
            if name and name in model.materials and 0 <= eid < n_el:
                m = model.materials[name]
                props[eid, 0] = m.youngs_modulus
                props[eid, 1] = m.poissons_ratio
    return props


def _mesh_node(model: FEAModel, node_id: int, is_geometry_node: bool) -> int | None:
    if is_geometry_node and model.geometry_to_mesh_node_map:
        return model.geometry_to_mesh_node_map.get(node_id)
    return node_id


def solid_load_vector(model: FEAModel) -> np.ndarray:
    """3-DOF/node load vector from ``LoadDef.fx/fy/fz`` (solid_solver.py:87-93)."""
    n = len(model.mesh_nodes)
    F = np.zeros(3 * n, dtype=np.float64)
    if not model.loads:
        return F
    ids = np.array([ld.node_id for ld in model.loads], dtype=np.int64)
    f = np.array([[ld.fx, ld.fy, ld.fz] for ld in model.loads], dtype=np.float64)
    ok = ids < n
    np.add.at(F.reshape(-1, 3), ids[ok], f[ok])
    return F


def solid_fixed_dofs(model: FEAModel) -> np.ndarray:
    """Global indices of FIXED translational DOFs, in support order (solid_solver.py:96-103)."""
    n = len(model.mesh_nodes)
    out: list[int] = []
    for s in model.supports:
        nid = s.node_id
        if nid < n:
            for local, c in enumerate(s.constraints[:3]):
                if c.dof_type == DOFType.FIXED:
                    out.append(nid * 3 + local)
    return np.asarray(out, dtype=np.int64)
