"""Host-side occupant registries: one row per occupant.

The reference registers each occupant once (``MATERIAL_MODELS`` in
src/components/materials/index.ts, ``LIGHT_KINDS`` in src/components/lights/index.ts, the
primitives of src/components/intersection/index.ts) and generates everything else from
those rows.  Here a surface material model is a device header under
``csrc/device/materials/`` (its struct and one line in ``materials/registry.cuh``) plus a
row below, which tells the compiler how to pack its record and the adjoint which of its
parameters are live; a light kind is a header under ``csrc/device/lights/`` plus a row that
packs its light record.  A row's id is the C ABI's ``PTR_MAT_*`` / ``PTR_LIGHT_*`` constant,
the struct's ``kId``; ``tests/test_occupants.py`` checks that the registries agree.
"""
import math
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


def _quad_record(l):
    """lights/quad/quad.ts: corner, edges, unit normal and area."""
    corner, e1, e2 = l["corner"], l["edge1"], l["edge2"]
    c = [e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]]
    area = math.sqrt(c[0] ** 2 + c[1] ** 2 + c[2] ** 2)
    nrm = [c[0] / area, c[1] / area, c[2] / area]
    geo = list(corner) + list(e1) + list(e2) + nrm
    return geo + [area], geo, area


def _sphere_record(l):
    """lights/sphere/sphere.ts: centre and radius."""
    geo = list(l.get("position", l.get("center"))) + [l["radius"]]
    return geo, geo, float(l["radius"])


def _point_record(l):
    """lights/point/point.ts: position only (a delta light)."""
    return list(l["position"]), None, None


@dataclass(frozen=True)
class LightKind:
    """A light kind.

    name         the scene format's light ``kind`` string
    kind         ptr_light.kind (abi.LIGHT_*)
    header       its device header under csrc/device/lights/
    record       light dict -> (ptr_light.p values, the region's p values or None, the
                 power geometry: area, radius or None); None for kinds not authored as
                 light records
    region_shape an authored light of this kind is also a hittable region of this shape
                 (with a synthesized emissive material), or None
    thin         that region's thin flag
    """
    name: str
    kind: int
    header: str
    record: object = None
    region_shape: int = None
    thin: int = 0


LIGHT_KIND_ROWS = {k.name: k for k in (
    LightKind("quad", abi.LIGHT_QUAD, "quad.cuh", _quad_record, abi.SHAPE_QUAD, thin=1),
    LightKind("sphere", abi.LIGHT_SPHERE, "sphere.cuh", _sphere_record, abi.SHAPE_SPHERE),
    LightKind("point", abi.LIGHT_POINT, "point.cuh", _point_record),
    # an emissive mesh object's light (lights/mesh/mesh.ts): never an authored record
    LightKind("mesh", abi.LIGHT_MESH, "mesh.cuh"),
)}
LIGHT_BY_ID = {k.kind: k for k in LIGHT_KIND_ROWS.values()}
# the kinds a scene may author as light records: name -> abi id
LIGHT_KINDS = {k.name: k.kind for k in LIGHT_KIND_ROWS.values() if k.record is not None}

PRIMITIVES = {"plane": abi.SHAPE_PLANE, "sphere": abi.SHAPE_SPHERE, "quad": abi.SHAPE_QUAD,
              "box": abi.SHAPE_BOX}
