"""Host-side occupant registries: one row per occupant.

The reference registers each occupant once (``MATERIAL_MODELS`` in
src/components/materials/index.ts, ``LIGHT_KINDS`` in src/components/lights/index.ts, the
primitives of src/components/intersection/index.ts) and generates everything else from
those rows.  Here a surface material model is a device header under
``csrc/device/materials/`` (its struct and one line in ``materials/registry.cuh``) plus the
row below, which tells the compiler how to pack its record and the adjoint which of its
parameters are live.  Its ``model`` value is the C ABI's ``PTR_MAT_*`` constant, the struct's
``kModel``; ``tests/test_occupants.py`` checks that both registries list the same models.
"""
from dataclasses import dataclass

from . import abi


@dataclass(frozen=True)
class MaterialModel:
    """A surface material model.

    name        the scene format's ``model`` string
    model       ptr_material.model (abi.MAT_*)
    header      its device header under csrc/device/materials/
    ior         its regions' IOR row comes from the material's ``ior`` (default 1.5)
    emitter     its ``emission`` makes the surface an emitter (light records, MIS)
    grad_color  the ptr_material field the adjoint's colour slots differentiate, or None
    grad_alpha  the adjoint differentiates its GGX alpha
    grad_ior    the adjoint differentiates its IOR (interface terms; live when a region uses it)
    """
    name: str
    model: int
    header: str
    ior: bool = False
    emitter: bool = False
    grad_color: str = None
    grad_alpha: bool = False
    grad_ior: bool = False


MATERIAL_MODELS = {m.name: m for m in (
    MaterialModel("lambert", abi.MAT_LAMBERT, "lambert.cuh", emitter=True, grad_color="albedo"),
    MaterialModel("dielectric", abi.MAT_DIELECTRIC, "dielectric.cuh", ior=True, grad_color="transmittance",
                  grad_ior=True),
    MaterialModel("ggx", abi.MAT_GGX, "ggx.cuh", grad_color="f0", grad_alpha=True),
    MaterialModel("mirror", abi.MAT_MIRROR, "mirror.cuh", grad_color="f0"),
    MaterialModel("none", abi.MAT_NONE, "null.cuh"),
    MaterialModel("rough_dielectric", abi.MAT_ROUGH_DIELECTRIC, "rough_dielectric.cuh", ior=True),
)}

# ptr_material.model -> row
MATERIAL_BY_ID = {m.model: m for m in MATERIAL_MODELS.values()}

PRIMITIVES = {"plane": abi.SHAPE_PLANE, "sphere": abi.SHAPE_SPHERE, "quad": abi.SHAPE_QUAD,
              "box": abi.SHAPE_BOX}
LIGHT_KINDS = {"quad": abi.LIGHT_QUAD, "sphere": abi.LIGHT_SPHERE, "point": abi.LIGHT_POINT}
