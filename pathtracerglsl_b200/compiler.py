"""SceneDescription + RenderStrategy -> CompiledRenderer + packed scene data.

Host mirror of the reference's Compiler for the transport-loop path
(``src/compiler/Compiler.ts:14-72``: Analyze -> Validate -> Plan -> Generate).  The
"Generate" stage here emits no shader text: it packs the plan into the flat tables of
``include/ptx_rt.h`` that the CUDA kernels read (the unrolled arms the GLSL emitter bakes
as literals become table rows), plus a ``ptr_program_desc`` with the estimator knobs.

Inputs use the reference's own JSON shapes (``src/compiler/types.ts:21-721``): objects
``{type, parameters, material}``, materials ``{model, albedo, emission, ior, roughness,
f0, medium}``, lights ``{kind, emission, ...}``, ``environment``, ``ambientMedium``,
strategies ``{id, measurement, estimator, view}``.  Errors are collected in a
DiagnosticBag and raised together (``src/errors/DiagnosticBag.ts:310`` throwIfErrors).
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi
from . import field as medium_field
from . import occupants

# ----------------------------------------------------------------------------- diagnostics


class Diagnostic:
    def __init__(self, severity, code, message):
        self.severity, self.code, self.message = severity, code, message

    def __repr__(self):
        return f"{self.severity}[{self.code}]: {self.message}"


class CompileError(Exception):
    """All errors of one compile, like ``DiagnosticBag.throwIfErrors``."""

    def __init__(self, diagnostics):
        self.diagnostics = diagnostics
        super().__init__("; ".join(f"[{d.code}] {d.message}" for d in diagnostics))


class DiagnosticBag:
    def __init__(self):
        self.items = []

    def error(self, code, message):
        self.items.append(Diagnostic("error", code, message))

    def warning(self, code, message):
        self.items.append(Diagnostic("warning", code, message))

    @property
    def errors(self):
        return [d for d in self.items if d.severity == "error"]

    @property
    def warnings(self):
        return [d for d in self.items if d.severity == "warning"]

    def throw_if_errors(self):
        if self.errors:
            raise CompileError(self.errors)


# ----------------------------------------------------------------------------- values

def is_param(v):
    return isinstance(v, dict) and "param" in v


def _has_param(v):
    if is_param(v):
        return True
    if isinstance(v, (list, tuple)):
        return any(_has_param(x) for x in v)
    if isinstance(v, dict):
        return any(_has_param(x) for x in v.values())
    return False


def resolve(v, params, default=None):
    """``Value<T>`` -> concrete value: constants as is, ``{param}`` from ``params`` or
    its default (contracts §2.8 in the reference's types.ts:257-275)."""
    if v is None:
        return default
    if is_param(v):
        return params.get(v["param"], v.get("default", default))
    return v


_BUNDLED_SPECTRAL = None


def _bundled_spectral():
    global _BUNDLED_SPECTRAL
    if _BUNDLED_SPECTRAL is None:
        from .spectral import SpectralModel
        _BUNDLED_SPECTRAL = SpectralModel.bundled()
    return _BUNDLED_SPECTRAL


def is_blackbody(v):
    return isinstance(v, dict) and "blackbody" in v


def rgb(v, params, default):
    """A SpectrumProperty as RGB: scalars broadcast (types.ts SpectrumProperty); a
    ``{blackbody: {kelvin, scale}}`` emission becomes its RGB stand-in, the unit-Y Planck
    colour times scale (spectra/blackbody/blackbody.ts blackbodyRGB)."""
    v = resolve(v, params, default)
    if v is None:
        v = default
    if isinstance(v, (int, float)):
        return [float(v)] * 3
    if is_blackbody(v):
        b = v["blackbody"]
        return _bundled_spectral().blackbody_rgb(float(resolve(b.get("kelvin"), params, 6500.0)),
                                                 float(resolve(b.get("scale"), params, 1.0)))
    if isinstance(v, dict):
        raise ValueError(f"unsupported spectrum value {v!r}")
    return [float(x) for x in v]


def _f32(x):
    return float(np.float32(x))


def _norm3(v):
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return [v[0] / n, v[1] / n, v[2] / n]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def camera_basis(position, target):
    """``cameraBasis`` (src/components/camera/basis.ts:49-55), float64 like the TS."""
    fwd = _norm3([target[i] - position[i] for i in range(3)])
    up_ref = [0.0, 0.0, 1.0] if abs(fwd[1]) > 0.999999 else [0.0, 1.0, 0.0]
    right = _norm3(_cross(fwd, up_ref))
    up = _cross(right, fwd)
    return fwd, right, up


# ----------------------------------------------------------------------------- registries
# The occupant registries (one row per occupant, like the reference's MATERIAL_MODELS /
# LIGHT_KINDS / PRIMITIVES registries) live in occupants.py.
MATERIAL_MODELS = occupants.MATERIAL_MODELS
PRIMITIVES = occupants.PRIMITIVES
LIGHT_KINDS = occupants.LIGHT_KINDS
DIRECT = {"none": abi.DIRECT_NONE, "nee": abi.DIRECT_NEE, "mis": abi.DIRECT_MIS}
# meshTraversal 'bvh' / 'cwbvh'; instanceAccel 'tlas' / 'cwbvh' ('linear', the reference's
# scan over every instance, returns the same nearest hit: it walks the binary TLAS here)
ACCELS = {"bvh": abi.ACCEL_BVH, "tlas": abi.ACCEL_BVH, "linear": abi.ACCEL_BVH, "cwbvh": abi.ACCEL_CWBVH}
THIN_SHAPES = {"quad"}


# ----------------------------------------------------------------------------- outputs

@dataclass
class PackedScene:
    """The scene-data plan, executed: every table the device reads, host-owned."""
    regions: np.ndarray
    materials: np.ndarray
    lights: np.ndarray
    ambient_material: int
    env: dict
    meshes: list = field(default_factory=list)
    batches: list = field(default_factory=list)
    region_names: list = field(default_factory=list)
    material_names: list = field(default_factory=list)
    spectral: object = None     # spectral.SpectralTables of spectral strategies, else None
    light_tree: object = None   # float32 nodes (8 per node) under light-tree selection, else None
    light_trails: object = None # uint32 trail words (2 per light)
    field_code: object = None   # uint32 programs of heterogeneous media coefficients

    def desc(self):
        """A ``ptr_scene_desc`` pointing into this object's arrays (keep self alive)."""
        d = abi.SceneDesc()
        d.abi_version = abi.ABI_VERSION
        d.n_regions = len(self.regions)
        d.regions = self.regions.ctypes.data_as(abi.C.POINTER(abi.Region))
        d.n_materials = len(self.materials)
        d.materials = self.materials.ctypes.data_as(abi.C.POINTER(abi.Material))
        d.n_lights = len(self.lights)
        d.lights = self.lights.ctypes.data_as(abi.C.POINTER(abi.Light)) if len(self.lights) else None
        d.ambient_material = self.ambient_material
        e = self.env
        d.env.kind = e["kind"]
        d.env.sample_as_light = int(e.get("sample_as_light", 0))
        d.env.color = abi.F4(*(list(e.get("color", [0, 0, 0])) + [0.0]))
        d.env.intensity = e.get("intensity", 1.0)
        d.env.select_prob = e.get("select_prob", 1.0)
        d.env.rotation = e.get("rotation", 0.0)
        if e["kind"] == abi.ENV_IMAGE:
            d.env.width, d.env.height = e["width"], e["height"]
            d.env.radiance = e["radiance"].ctypes.data_as(abi.C.POINTER(abi.C.c_float))
            d.env.marginal = e["marginal"].ctypes.data_as(abi.C.POINTER(abi.C.c_float))
            d.env.conditional = e["conditional"].ctypes.data_as(abi.C.POINTER(abi.C.c_float))
        if self.meshes:
            self._mesh_arr = (abi.MeshDesc * len(self.meshes))()
            for i, m in enumerate(self.meshes):
                md = self._mesh_arr[i]
                md.n_vertices = len(m["positions"]) // 3
                md.n_triangles = len(m["indices"]) // 3
                md.positions = m["positions"].ctypes.data_as(abi.C.POINTER(abi.C.c_float))
                md.indices = m["indices"].ctypes.data_as(abi.C.POINTER(abi.C.c_uint32))
                ta = m.get("tri_alpha")
                md.tri_alpha = ta.ctypes.data_as(abi.C.POINTER(abi.C.c_float)) if ta is not None else None
            d.n_meshes = len(self.meshes)
            d.meshes = self._mesh_arr
        if self.batches:
            self._batch_arr = (abi.BatchDesc * len(self.batches))()
            for i, b in enumerate(self.batches):
                bd = self._batch_arr[i]
                bd.prototype_shape = b["prototype_shape"]
                bd.prototype_ref = b.get("prototype_ref", -1)
                bd.n_instances = len(b["placements"]) // 8
                bd.proto = abi.F4(*b.get("proto", [0, 0, 0, 0]))
                bd.light_base = b.get("light_base", -1)
                bd.placements = b["placements"].ctypes.data_as(abi.C.POINTER(abi.C.c_float))
            d.n_batches = len(self.batches)
            d.batches = self._batch_arr
        if self.spectral is not None:
            self._spec_desc = self.spectral.desc()
            d.spectral = abi.C.pointer(self._spec_desc)
        if self.field_code is not None:
            d.n_field_code = len(self.field_code)
            d.field_code = self.field_code.ctypes.data_as(abi.C.POINTER(abi.C.c_uint32))
        if self.light_tree is not None:
            d.n_tree_nodes = len(self.light_tree) // 8
            d.light_tree = self.light_tree.ctypes.data_as(abi.C.POINTER(abi.C.c_float))
            d.light_trails = self.light_trails.ctypes.data_as(abi.C.POINTER(abi.C.c_uint32))
        return d


@dataclass
class CompiledRenderer:
    """The CompiledRenderer contract (src/compiler/types.ts:1084-1136) for this engine:
    the program description replaces ``shaders``/``pipeline``; ``uniforms`` are the
    host-side compute closures (camera basis, tan(fov/2), aspect)."""
    id: str
    program: abi.ProgramDesc
    strategy: dict
    parameters: dict
    export_targets: dict
    measurement: dict = None   # the strategy's measurement with every default filled in

    def camera(self, params, width, height):
        """Evaluate the camera uniforms (features/camera.ts:69-160) into a ``ptr_camera``."""
        p = {k: v["default"] for k, v in self.parameters.items()}
        p.update(params or {})
        pos, tgt, fov = p["camera.position"], p["camera.target"], p["camera.fov"]
        fwd, right, up = camera_basis(pos, tgt)
        cam = abi.Camera()
        cam.position = (abi.C.c_float * 3)(*pos)
        cam.forward = (abi.C.c_float * 3)(*fwd)
        cam.right = (abi.C.c_float * 3)(*right)
        cam.up = (abi.C.c_float * 3)(*up)
        cam.tan_fov = math.tan(fov / 2.0)
        cam.aspect = width / height if height else 1.0
        return cam


@dataclass
class CompiledScene:
    renderers: list
    scene_data: PackedScene
    warnings: list


# ----------------------------------------------------------------------------- compiler

class Compiler:
    """``Compiler.compile`` / ``compileScene`` (src/compiler/Compiler.ts:14-72).

    ``spectral_model``: the spectral colour model spectral strategies lift colours with
    (``spectral.SpectralModel``; default: the package's bundled subset)."""

    def __init__(self, spectral_model=None):
        self.spectral_model = spectral_model

    def compile(self, scene, strategy, params=None):
        out = self.compile_scene(scene, [strategy], params)
        return out.renderers[0], out.scene_data

    def compile_scene(self, scene, strategies, params=None):
        params = dict(params or {})
        bag = DiagnosticBag()
        for st in strategies:
            self._validate(scene, st, bag)
        bag.throw_if_errors()
        data = self._pack(scene, strategies, params, bag)
        bag.throw_if_errors()
        renderers = [self._program(scene, st, data) for st in strategies]
        return CompiledScene(renderers, data, bag.warnings)

    # -- Validate (src/compiler/analyze/Validator.ts:50) ------------------------------
    def _validate(self, scene, st, bag):
        mats = scene.get("materials", {})
        for i, o in enumerate(scene.get("objects", [])):
            kind = o.get("kind")
            if kind == "mesh":
                if "positions" not in o or "indices" not in o:
                    bag.error("invalid-mesh", f"object {i}: mesh needs positions and indices")
            elif kind == "instanced":
                proto = o.get("prototype", {})
                if proto.get("kind") != "mesh" and proto.get("type") != "sphere":
                    bag.error("unsupported", f"object {i}: instanced prototype must be a mesh or a sphere")
            elif o.get("type") not in PRIMITIVES:
                bag.error("unknown-primitive", f"object {i}: unknown primitive type {o.get('type')!r} "
                          f"(available: {', '.join(PRIMITIVES)})")
            mname = o.get("material") if kind != "instanced" else o.get("prototype", {}).get("material")
            if mname not in mats:
                bag.error("unknown-material", f"object {i}: unknown material {mname!r}")
        for name, m in mats.items():
            if m.get("model") not in MATERIAL_MODELS:
                bag.error("unknown-model", f"material {name!r}: unknown model {m.get('model')!r} "
                          f"(available: {', '.join(MATERIAL_MODELS)})")
        for i, l in enumerate(scene.get("lights", [])):
            if l.get("kind") == "mesh":
                # lights/mesh/mesh.ts validateAuthored: the only route is an emissive mesh object
                bag.error("unknown-light", f"light {i}: mesh lights are not authored as light records; set "
                          "`sampleAsLight` (or leave it on) on an emissive material used by a mesh object")
            elif l.get("kind") not in LIGHT_KINDS:
                bag.error("unknown-light", f"light {i}: unknown kind {l.get('kind')!r}")
        env = scene.get("environment", {"type": "none"})
        if env.get("type") not in ("none", "constant", "image", "procedural"):
            bag.error("unknown-environment", f"unknown environment type {env.get('type')!r}")
        am = scene.get("ambientMedium")
        if am is not None and am not in mats:
            bag.error("unknown-material", f"ambientMedium {am!r} is not a material")
        meas = st.get("measurement", {})
        est = st.get("estimator", {})
        mb = meas.get("maxBounces")
        if not isinstance(mb, int) or mb < 0:
            bag.error("invalid-setting", f"strategy {st.get('id')}: maxBounces must be a non-negative integer")
        if est.get("directLighting", "none") not in DIRECT:
            bag.error("invalid-setting", f"strategy {st.get('id')}: directLighting {est.get('directLighting')!r}")
        rr = est.get("russianRoulette")
        if rr is not None:
            ms = rr.get("maxSurvival", 0.95)
            if not (0.0 < ms <= 1.0):
                bag.error("invalid-setting", "russianRoulette.maxSurvival must be in (0, 1]")
        color = meas.get("color", "rgb")
        if color not in ("rgb", "spectral"):
            bag.error("invalid-setting", f"measurement.color {color!r} (available: rgb, spectral)")
        if color == "spectral":
            if scene.get("environment", {}).get("type", "none") not in ("none", "constant"):
                bag.error("unsupported", "spectral rendering supports constant environments only")
            if est.get("wavelengths", "visible") not in ("visible", "uniform"):
                bag.error("invalid-setting", f"estimator.wavelengths {est.get('wavelengths')!r} (available: visible, uniform)")
            lo, hi = meas.get("wavelengthRange", [360.0, 830.0])
            if not (360.0 <= lo < hi <= 830.0):
                bag.error("invalid-setting", "measurement.wavelengthRange must lie in [360, 830] nm")
        vs = est.get("volumeSampling", "analytic")
        if vs not in ("analytic", "delta-tracking", None):
            bag.error("unsupported", f"volumeSampling {vs!r} is not available in this build")
        for name, m in mats.items():
            med = m.get("medium") or {}
            het = [k for k in ("sigma_a", "sigma_s") if medium_field.is_field(med.get(k))]
            if not het:
                continue
            # Validator.ts:320-360: expression coefficients need a finite positive majorant
            maj = med.get("majorant")
            if not (isinstance(maj, (int, float)) and math.isfinite(maj) and maj > 0):
                bag.error("invalid-medium", f"Material '{name}': medium.{het[0]} is a GLSL expression but the medium "
                          "declares no majorant; heterogeneous media require a density ceiling (majorant: <finite number > 0>)")
            if meas.get("color", "rgb") == "spectral":
                bag.error("unsupported", f"Material '{name}': heterogeneous media render in RGB only in this build")
            if est.get("mediumLightSampling", "vertex") == "equiangular":
                bag.error("unsupported", f"Material '{name}': equiangular sampling through heterogeneous media is not available")
            for k in het:
                try:
                    medium_field.compile_field(med[k], {})
                except medium_field.FieldError as e:
                    bag.error("invalid-medium", f"Material '{name}': medium.{k}: {e}")
        aovs = meas.get("aovs") or []
        if any(a not in ("albedo", "normal") for a in aovs) or len(set(aovs)) != len(aovs):
            bag.error("invalid-setting", f"measurement.aovs {aovs!r}: each of albedo, normal at most once")
        if aovs and meas.get("color", "rgb") == "spectral":
            bag.error("unsupported", "measurement.aovs are RGB only")
        sel = est.get("lightSelection", "power")
        if sel not in ("power", "uniform", "bvh"):
            bag.error("invalid-setting", f"estimator.lightSelection {sel!r} (available: power, uniform, bvh)")
        if sel == "bvh":
            # Validator.ts:629-665: the tree needs constant emission and keeps equiangular
            # on the CDF path
            if est.get("mediumLightSampling", "vertex") == "equiangular":
                bag.error("unsupported", "estimator.lightSelection 'bvh' with mediumLightSampling 'equiangular' "
                          "is reserved; use 'vertex'")
            driven = [l.get("kind") for l in scene.get("lights", []) if _has_param(l.get("emission"))]
            driven += [n for n, m in mats.items() if _has_param(m.get("emission"))]
            if driven:
                bag.error("unsupported", "estimator.lightSelection 'bvh' requires constant light emission "
                          f"(driven: {', '.join(map(str, driven))}); use 'power'")
        mls = est.get("mediumLightSampling", "vertex")
        if mls not in ("vertex", "equiangular"):
            bag.error("invalid-setting", f"mediumLightSampling {mls!r} (available: vertex, equiangular)")
        if mls == "equiangular":
            # Validator.ts:506-540: equiangular is pinned to delta lights and plain NEE.  The
            # strategy key 'equiangularAreaLights' (this library's extension, not in the
            # reference) also admits quad and sphere lights.
            if est.get("directLighting") != "nee":
                bag.error("invalid-setting", "mediumLightSampling 'equiangular' requires directLighting 'nee'")
            area_ok = bool(est.get("equiangularAreaLights", False))
            kinds = ("point", "quad", "sphere") if area_ok else ("point",)
            if any(l.get("kind") not in kinds for l in scene.get("lights", [])):
                bag.error("invalid-setting", "mediumLightSampling 'equiangular' supports delta (point) lights only"
                          if not area_ok else "mediumLightSampling 'equiangular' supports point, quad and sphere lights")
            if not scene.get("lights"):
                bag.error("invalid-setting", "mediumLightSampling 'equiangular' needs at least one light")
            if meas.get("scattering") == "ignored":
                bag.error("invalid-setting", "mediumLightSampling 'equiangular' requires scattering media")
        for key in ("meshTraversal", "instanceAccel"):
            v = est.get(key)
            if v is not None and v not in ACCELS:
                bag.error("invalid-setting", f"{key} {v!r} (available: {', '.join(ACCELS)})")

    # -- Plan + pack (src/compiler/plan/Planner.ts:72, app/sceneData.ts:27) -----------
    def _pack(self, scene, strategies, params, bag):
        mats_src = scene.get("materials", {})
        mat_names = list(mats_src.keys())
        mat_index = {n: i for i, n in enumerate(mat_names)}
        materials = []
        self._field_code = []
        spec_src = []          # per material: the authored material, or a light's raw emission
        for n in mat_names:
            materials.append(self._material(mats_src[n], params))
            spec_src.append(("material", mats_src[n]))

        regions, region_names, lights = [], [], []
        meshes, batches = [], []
        for i, o in enumerate(scene.get("objects", [])):
            kind = o.get("kind")
            if kind == "mesh":
                r = abi.Region()
                r.shape = abi.SHAPE_MESH
                r.material = mat_index[o["material"]]
                r.thin = 0 if o.get("closed") else 1
                r.ref = len(meshes)
                meshes.append(self._mesh(o))
                r.ior = self._ior(mats_src[o["material"]], params)
            elif kind == "instanced":
                r = abi.Region()
                r.shape = abi.SHAPE_INSTANCES
                proto = o["prototype"]
                r.material = mat_index[proto["material"]]
                r.ref = len(batches)
                r.ior = self._ior(mats_src[proto["material"]], params)
                b = {"placements": self._placements(o["placements"])}
                if proto.get("kind") == "mesh":
                    b["prototype_shape"] = abi.SHAPE_MESH
                    b["prototype_ref"] = len(meshes)
                    meshes.append(self._mesh(proto))
                    r.thin = 1
                else:
                    pp = proto["parameters"]
                    b["prototype_shape"] = abi.SHAPE_SPHERE
                    b["proto"] = list(pp.get("center", [0, 0, 0])) + [pp["radius"]]
                    r.thin = 0
                batches.append(b)
            else:
                r = self._primitive(o, params)
                r.material = mat_index[o["material"]]
                r.ior = self._ior(mats_src[o["material"]], params)
            regions.append(r)
            region_names.append(o.get("name") or f"object_{i}")

        # Light roster (plan/dataTenants.ts lightRosterOf): authored lights, then emissive
        # analytic objects in scene order.  Authored area lights desugar into a hittable
        # region with a synthesized emissive material (impl-plan-area-lights A3).
        for li, l in enumerate(scene.get("lights", [])):
            kind = l["kind"]
            e = rgb(l.get("emission"), params, [1.0, 1.0, 1.0])
            rec = abi.Light()
            rec.kind = LIGHT_KINDS[kind]
            rec.radiance = abi.F4(*(e + [0.0]))
            rec.region = -1
            row = occupants.LIGHT_KIND_ROWS[kind]
            vals, region_p, geom = row.record(l)
            rec.p = (abi.C.c_float * 16)(*vals)
            if row.region_shape is not None:
                materials.append(self._light_material(e))
                spec_src.append(("light", l.get("emission", 1.0)))
                reg = abi.Region()
                reg.shape = row.region_shape
                reg.thin = row.thin
                reg.material = len(materials) - 1
                reg.ior = 1.0
                reg.p = (abi.C.c_float * 15)(*region_p)
                rec.region = len(regions)
                regions.append(reg)
                region_names.append(f"light_{li}")
            lights.append((rec, kind, e, geom, l.get("emission", 1.0)))
        for i, o in enumerate(scene.get("objects", [])):
            if o.get("kind") not in (None, "mesh"):
                continue
            m = mats_src[o["material"]]
            if m.get("sampleAsLight") is False or not getattr(MATERIAL_MODELS.get(m.get("model")), "emitter", False):
                continue
            e = rgb(m.get("emission"), params, [0.0, 0.0, 0.0])
            if max(e) <= 0.0 or (o.get("kind") is None and o["type"] not in ("sphere", "quad")):
                continue
            rec = abi.Light()
            rec.region = i
            rec.radiance = abi.F4(*(e + [0.0]))
            reg = regions[i]
            pp = o.get("parameters", {})
            if o.get("kind") == "mesh":
                # lights/mesh/mesh.ts: one-sided uniform area over the whole mesh; the world
                # total area (meshWorldArea, float64 over the float32 vertices) is the one
                # constant of its density and of its power pi * A * Le
                mesh = meshes[reg.ref]
                area = _mesh_area(mesh["positions"], mesh["indices"])
                if not area > 0.0:
                    continue
                rec.kind = abi.LIGHT_MESH
                vals = [float(reg.ref)] + [0.0] * 11 + [area]
                rec.p = (abi.C.c_float * 16)(*vals)
                geom = area
                lights.append((rec, "mesh", e, geom, m.get("emission")))
                continue
            if o["type"] == "sphere":
                rec.kind = abi.LIGHT_SPHERE
                rec.p = (abi.C.c_float * 16)(*(list(reg.p[0:4])))
                geom = float(pp["radius"]) * float((o.get("transform") or {}).get("scale", 1.0))
            else:
                rec.kind = abi.LIGHT_QUAD
                c = _cross(pp["edge1"], pp["edge2"])
                area = math.sqrt(c[0] ** 2 + c[1] ** 2 + c[2] ** 2)
                rec.p = (abi.C.c_float * 16)(*(list(reg.p[0:12]) + [area]))
                geom = area
            lights.append((rec, o["type"], e, geom, m.get("emission")))

        sel_mode = "power"
        tree_direct = False
        for st in strategies:
            sel_mode = st.get("estimator", {}).get("lightSelection", "power")
            tree_direct = st.get("estimator", {}).get("directLighting", "none") != "none"
        if sel_mode == "bvh" and tree_direct:
            # instanced emitters (dataTenants.ts batchLightEligible): a sphere-prototype batch
            # with a constant emissive Lambert material makes every instance a sphere light
            # of the tree, in placement order from the batch's light_base
            for i, o in enumerate(scene.get("objects", [])):
                if o.get("kind") != "instanced":
                    continue
                proto = o["prototype"]
                m = mats_src[proto["material"]]
                if proto.get("kind") == "mesh" or proto.get("type") != "sphere":
                    continue
                if m.get("sampleAsLight") is False or not getattr(MATERIAL_MODELS.get(m.get("model")), "emitter", False):
                    continue
                e = rgb(m.get("emission"), params, [0.0, 0.0, 0.0])
                if max(e) <= 0.0:
                    continue
                b = batches[regions[i].ref]
                b["light_base"] = len(lights)
                cen, rad = _instance_spheres(b["placements"], b["proto"])
                for k in range(len(rad)):
                    rec = abi.Light()
                    rec.kind = abi.LIGHT_SPHERE
                    rec.region = -1
                    rec.radiance = abi.F4(*(e + [0.0]))
                    rec.p = (abi.C.c_float * 16)(float(cen[k, 0]), float(cen[k, 1]), float(cen[k, 2]), float(rad[k]))
                    lights.append((rec, "sphere", e, float(rad[k]), m.get("emission")))

        # Selection CDF (features/lighting.ts computeSelectPdf; power per kind from the
        # descriptors: quad pi*A*Le, sphere pi*4*pi*r^2*Le, point 4*pi*I).
        weights = [1.0 if sel_mode == "uniform" else _light_power(rec.kind, e, geom)
                   for rec, kind, e, geom, _raw in lights]
        total = sum(weights)
        acc = 0.0
        light_arr = np.zeros(len(lights), dtype=np.dtype((np.void, abi.C.sizeof(abi.Light))))
        light_recs = (abi.Light * max(len(lights), 1))()
        for i, (rec, kind, e, geom, _raw) in enumerate(lights):
            pdf = weights[i] / total
            acc += pdf
            rec.select_pdf = pdf
            rec.select_cdf = acc
            light_recs[i] = rec
        light_arr = np.frombuffer(bytes(light_recs), dtype=np.uint8).reshape(max(len(lights), 1), -1)[:len(lights)].copy()
        tree = trails = None
        if sel_mode == "bvh" and tree_direct and lights:
            tree, trails = _light_tree([rec for rec, *_x in lights],
                                       [_light_power(rec.kind, e, geom) for rec, kind, e, geom, _raw in lights],
                                       meshes)

        env = self._environment(scene.get("environment") or {"type": "none"}, params, scene, lights, bag)
        if tree is not None and "select_prob" in env:
            env["select_prob"] = 0.5   # lighting.ts:476-481: the env against the whole tree
        am = scene.get("ambientMedium")
        packed = PackedScene(
            regions=_as_bytes(regions, abi.Region),
            materials=_as_bytes([m for m in materials], abi.Material),
            lights=light_arr,
            ambient_material=mat_index[am] if am is not None else -1,
            env=env, meshes=meshes, batches=batches,
            region_names=region_names, material_names=mat_names,
            light_tree=tree, light_trails=trails,
            field_code=np.asarray(self._field_code, np.uint32) if self._field_code else None,
        )
        if any(st.get("measurement", {}).get("color", "rgb") == "spectral" for st in strategies):
            packed.spectral = self._spectral_tables(spec_src, [raw for *_x, raw in lights],
                                                    scene.get("environment") or {"type": "none"}, params)
        return packed

    # -- the spectral colour model: every constant colour lifted once (lookup.glsl:38-59)
    def _spectral_tables(self, spec_src, light_raw, env, params):
        model = self.spectral_model or _bundled_spectral()

        def emission(v, default):
            v = resolve(v, params, default)
            if is_blackbody(v):
                b = v["blackbody"]
                return model.blackbody(float(resolve(b.get("kelvin"), params, 6500.0)),
                                       float(resolve(b.get("scale"), params, 1.0)))
            return model.emission(rgb(v, params, default))

        mats = []
        for kind, src in spec_src:
            sm = abi.SpectralMaterial()
            if kind == "light":
                sm.albedo = model.reflectance([0.0, 0.0, 0.0])
                sm.emission = emission(src, 1.0)
                sm.transmittance = model.reflectance([1.0, 1.0, 1.0])
                sm.f0 = model.reflectance([0.9, 0.9, 0.9])
                sm.sigma_a = sm.sigma_s = model.coefficient([0.0, 0.0, 0.0])
            else:
                m = src
                sm.albedo = model.reflectance(rgb(m.get("albedo"), params, [0.8, 0.8, 0.8]))
                sm.emission = emission(m.get("emission"), [0.0, 0.0, 0.0])
                sm.transmittance = model.reflectance(rgb(m.get("transmittance"), params, [1.0, 1.0, 1.0]))
                sm.f0 = model.reflectance(rgb(m.get("f0"), params, [0.9, 0.9, 0.9]))
                med = m.get("medium") or {}
                sm.sigma_a = model.coefficient(rgb(med.get("sigma_a"), params, [0.0, 0.0, 0.0]))
                sm.sigma_s = model.coefficient(rgb(med.get("sigma_s"), params, [0.0, 0.0, 0.0]))
            mats.append(sm)
        lights = [emission(raw, 1.0) for raw in light_raw]
        env_spec = model.emission(rgb(env.get("color"), params, [1.0, 1.0, 1.0])) \
            if env.get("type") == "constant" else model.coefficient([0.0, 0.0, 0.0])
        return model.spectral_desc(mats, lights, env_spec)

    def _primitive(self, o, params):
        t = o["type"]
        p = o.get("parameters", {})
        r = abi.Region()
        r.shape = PRIMITIVES[t]
        r.thin = 1 if t in THIN_SHAPES else 0
        vals = []
        if t == "plane":
            n = p["normal"]
            ln = math.sqrt(sum(x * x for x in n))
            vals = [n[0] / ln, n[1] / ln, n[2] / ln, p.get("offset", 0.0) / ln]   # canonicalPlane
        elif t == "sphere":
            vals = list(p.get("center", [0, 0, 0])) + [p["radius"]]
        elif t == "quad":
            corner, e1, e2 = p["corner"], p["edge1"], p["edge2"]
            nrm = _norm3(_cross(e1, e2))
            vals = list(corner) + list(e1) + list(e2) + nrm
        elif t == "box":
            vals = list(p.get("center", [0, 0, 0])) + list(p["halfSize"])
        tr = o.get("transform")
        if tr:
            vals = self._fold_transform(t, vals, tr)
        r.p = (abi.C.c_float * 15)(*vals)
        return r

    @staticmethod
    def _fold_transform(t, vals, tr):
        """Fold a constant similarity into the canonical parameters (translation and
        uniform scale; the analytic set is similarity-closed, fable-transforms §5.1)."""
        if tr.get("rotation") is not None:
            raise CompileError([Diagnostic("error", "unsupported", "rotated primitives are not available in this build")])
        pos = tr.get("position", [0, 0, 0])
        s = float(tr.get("scale", 1.0))
        if t == "sphere":
            return [vals[0] * s + pos[0], vals[1] * s + pos[1], vals[2] * s + pos[2], vals[3] * s]
        if t == "box":
            return [vals[0] * s + pos[0], vals[1] * s + pos[1], vals[2] * s + pos[2]] + [v * s for v in vals[3:6]]
        if t == "quad":
            return [vals[i] * s + pos[i] for i in range(3)] + [v * s for v in vals[3:9]] + vals[9:12]
        if t == "plane":
            n = vals[0:3]
            return n + [vals[3] * s - (n[0] * pos[0] + n[1] * pos[1] + n[2] * pos[2])]
        return vals

    def _material(self, m, params):
        """MaterialProperties defaults of the generated lookup (features/materials.ts:372-423):
        albedo 0.8, emission 0, transmittance 1, f0 0.9, roughness 0.5."""
        rec = abi.Material()
        model = m["model"]
        row = MATERIAL_MODELS[model]
        rec.model = row.model
        alb = rgb(m.get("albedo"), params, [0.8, 0.8, 0.8])
        emi = rgb(m.get("emission"), params, [0.0, 0.0, 0.0])
        rec.albedo = abi.F4(*(alb + [0.0]))
        rec.emission = abi.F4(*(emi + [0.0]))
        rec.transmittance = abi.F4(*(rgb(m.get("transmittance"), params, [1.0, 1.0, 1.0]) + [0.0]))
        rec.f0 = abi.F4(*(rgb(m.get("f0"), params, [0.9, 0.9, 0.9]) + [0.0]))
        rough = float(resolve(m.get("roughness"), params, 0.5))
        rec.alpha = max(1e-3, rough * rough)          # ggx.glsl:7-9 derived row
        flags = 0
        if row.emitter and max(emi) > 0.0:
            flags |= abi.MATF_EMISSIVE
        med = m.get("medium")
        if med is not None:
            def coef(key, slot):
                v = med.get(key)
                if medium_field.is_field(v):   # heterogeneous: the stack program, 1 + its offset
                    code = getattr(self, "_field_code", None)
                    if code is None:
                        code = self._field_code = []
                    setattr(rec, slot, 1 + len(code))
                    code.extend(medium_field.compile_field(v, params))
                    return None
                return rgb(v, params, [0.0, 0.0, 0.0])
            sa = coef("sigma_a", "field_a")
            ss = coef("sigma_s", "field_s")
            rec.sigma_a = abi.F4(*((sa or [0.0] * 3) + [0.0]))
            rec.sigma_s = abi.F4(*((ss or [0.0] * 3) + [0.0]))
            rec.phase_g = float(resolve(med.get("phase_g", med.get("g")), params, 0.0))
            if rec.field_a or rec.field_s:
                rec.majorant = float(med["majorant"])
            flags |= abi.MATF_MEDIUM
            if ss is None or max(ss) > 0.0:
                flags |= abi.MATF_SCATTERING
        rec.flags = flags
        return rec

    @staticmethod
    def _light_material(e):
        rec = abi.Material()
        rec.model = abi.MAT_LAMBERT
        rec.albedo = abi.F4(0.0, 0.0, 0.0, 0.0)
        rec.emission = abi.F4(*(list(e) + [0.0]))
        rec.transmittance = abi.F4(1.0, 1.0, 1.0, 0.0)
        rec.f0 = abi.F4(0.9, 0.9, 0.9, 0.0)
        rec.alpha = 0.25
        rec.flags = abi.MATF_EMISSIVE
        return rec

    @staticmethod
    def _ior(m, params):
        row = MATERIAL_MODELS.get(m.get("model"))
        if row is not None and row.ior:   # the region-table ior row
            return float(resolve(m.get("ior"), params, 1.5))
        return 1.0

    @staticmethod
    def _mesh(o):
        pos = np.ascontiguousarray(np.asarray(o["positions"], np.float32).reshape(-1))
        idx = np.ascontiguousarray(np.asarray(o["indices"], np.uint32).reshape(-1))
        out = {"positions": pos, "indices": idx}
        if o.get("triangleAlpha") is not None:
            out["tri_alpha"] = np.ascontiguousarray(np.asarray(o["triangleAlpha"], np.float32))
        return out

    @staticmethod
    def _placements(pl):
        """Placement records (intersection/instancing/placement.glsl:19-41): the world ->
        rigid-frame quaternion q (xyzw) and ts = (t_rigid, s) with t_rigid = -R^T t."""
        recs = []
        for tr in pl:
            pos = tr.get("position", [0, 0, 0])
            s = float(tr.get("scale", 1.0))
            rot = tr.get("rotation")
            if rot is None:
                qx, qy, qz, qw = 0.0, 0.0, 0.0, 1.0
            elif isinstance(rot, dict):
                ax = _norm3(rot["axis"])
                h = rot["angle"] / 2.0
                qx, qy, qz, qw = ax[0] * math.sin(h), ax[1] * math.sin(h), ax[2] * math.sin(h), math.cos(h)
            else:
                qx, qy, qz, qw = rot
            # inverse rotation (conjugate) maps world to the rigid frame
            iq = (-qx, -qy, -qz, qw)
            t_r = _qrot(iq, [-pos[0], -pos[1], -pos[2]])
            recs.extend([iq[0], iq[1], iq[2], iq[3], t_r[0], t_r[1], t_r[2], s])
        return np.asarray(recs, np.float32)

    def _environment(self, env, params, scene, lights, bag):
        t = env.get("type", "none")
        if t == "none":
            return {"kind": abi.ENV_NONE}
        intensity = float(resolve(env.get("intensity"), params, 1.0))
        if t == "constant":
            col = rgb(env.get("color"), params, [1.0, 1.0, 1.0])
            sal = bool(env.get("sampleAsLight", False))
            out = {"kind": abi.ENV_CONSTANT, "color": col, "intensity": intensity,
                   "sample_as_light": sal, "rotation": 0.0}
            out["select_prob"] = self._env_select_prob(sum(col) / 3.0, intensity, scene, lights)
            return out
        # tabulated environments: an equirect RGB table (image, or a procedural recipe already
        # baked into one) + the importance CDFs; joins NEE/MIS by default (sampleAsLight true)
        table = env.get("table")
        if table is None:
            bag.error("invalid-environment", f"environment {t!r} needs a 'table' (H x W x 3 float32 equirect radiance)")
            return {"kind": abi.ENV_NONE}
        table = np.ascontiguousarray(np.asarray(table, np.float32))
        if table.ndim != 3 or table.shape[2] != 3 or not np.isfinite(table).all() or (table < 0).any():
            bag.error("invalid-environment", "environment table must be H x W x 3, finite and nonnegative")
            return {"kind": abi.ENV_NONE}
        H, W = table.shape[:2]
        cond, marg, total = build_env_importance(table)
        rgba = np.zeros((H, W, 4), np.float32)
        rgba[:, :, :3] = table
        sal = bool(env.get("sampleAsLight", True))
        out = {"kind": abi.ENV_IMAGE, "width": W, "height": H, "radiance": rgba.reshape(-1),
               "marginal": marg, "conditional": cond.reshape(-1), "intensity": intensity,
               "sample_as_light": sal, "rotation": float(resolve(env.get("rotation"), params, 0.0)),
               "total_weight": total}
        mean_l = (total * math.pi) / (2 * W * H)      # equirect: integral L dOmega / 4 pi
        out["select_prob"] = self._env_select_prob(mean_l, intensity, scene, lights)
        return out

    @staticmethod
    def _env_select_prob(mean_l, intensity, scene, lights):
        """envSelectionProbability (features/lighting.ts:488-525), 'power' selection."""
        r = 1.0
        for o in scene.get("objects", []):
            p = o.get("parameters", {})
            center = 0.0
            extent = 0.0
            for k in ("center", "corner"):
                if k in p:
                    center = max(center, math.hypot(*p[k]))
            for k in ("radius", "halfSize", "offset"):
                if k in p:
                    v = p[k]
                    extent += max(v) if isinstance(v, (list, tuple)) else float(v)
            r = max(r, center + extent)
        phi_env = 4 * math.pi * math.pi * r * r * mean_l * intensity
        phi_fin = sum(_light_power(rec.kind, e, geom) for rec, kind, e, geom, _raw in lights)
        return min(0.99, max(0.01, phi_env / max(phi_env + phi_fin, 1e-20)))

    # -- Generate: the program description (flags of plan/types.ts:39-112) -------------
    def _program(self, scene, st, data):
        meas = st.get("measurement", {})
        est = st.get("estimator", {})
        prog = abi.ProgramDesc()
        prog.abi_version = abi.ABI_VERSION
        prog.max_bounces = int(meas["maxBounces"])
        prog.max_null_crossings = int(meas.get("maxNullCrossings", 32))
        prog.direct = DIRECT[est.get("directLighting", "none")]
        rr = est.get("russianRoulette")
        prog.rr_start = int(rr.get("startDepth", 0)) if rr else -1
        prog.rr_max_survival = float(rr.get("maxSurvival", 0.95)) if rr else 1.0
        prog.scattering = 0 if meas.get("scattering") == "ignored" else 1
        prog.accel = ACCELS[est.get("meshTraversal") or "bvh"]                 # mesh BLAS walk
        prog.instance_accel = ACCELS[est.get("instanceAccel") or "tlas"]       # instanced batches' TLAS
        prog.color = abi.COLOR_SPECTRAL if meas.get("color", "rgb") == "spectral" else abi.COLOR_RGB
        prog.wavelengths = abi.WAVELENGTHS_UNIFORM if est.get("wavelengths") == "uniform" else abi.WAVELENGTHS_VISIBLE
        lo, hi = meas.get("wavelengthRange", [360.0, 830.0])
        prog.lambda_min, prog.lambda_max = float(lo), float(hi)
        prog.aovs = sum({"albedo": abi.AOV_ALBEDO, "normal": abi.AOV_NORMAL}[a] for a in set(meas.get("aovs") or []))
        prog.light_tree = int(est.get("lightSelection") == "bvh" and prog.direct != abi.DIRECT_NONE
                              and getattr(data, "light_tree", None) is not None)
        prog.equiangular = abi.EQUIANGULAR_OFF
        if est.get("mediumLightSampling") == "equiangular":
            prog.equiangular = abi.EQUIANGULAR_AREA if est.get("equiangularAreaLights") else abi.EQUIANGULAR_DELTA
        cam = meas.get("camera", {})
        fov = cam.get("fov", 0.8)
        fov_default = fov.get("default", 0.8) if is_param(fov) else fov
        parameters = {
            "camera.position": {"type": "vec3", "default": list(cam.get("position", [0, 0, 8]))},
            "camera.target": {"type": "vec3", "default": list(cam.get("target", [0, 0, 0]))},
            "camera.fov": {"type": "float", "default": fov_default},
        }
        rid = f"{st.get('id', 'strategy')}-{scene.get('id', 'scene')}"
        exports = {"radiance": {"format": "float"}, "variance": {"format": "float"}}
        for a in meas.get("aovs") or []:   # first-hit pictures (components/aov)
            exports[a] = {"format": "float"}
        return CompiledRenderer(rid, prog, st, parameters, exports, resolve_measurement(scene, st))


DEFAULT_MAX_NULL_CROSSINGS = 32
DEFAULT_SENSORS = {"rgb": "ideal", "spectral": "cie1931"}


def resolve_measurement(scene, strategy):
    """``resolveMeasurement`` (src/compiler/plan/measurement.ts:14-35): the strategy's
    measurement section with every default filled in, i.e. what the image estimates,
    truncations included.  The reproducibility stamp records it."""
    m = strategy.get("measurement", {})
    color = m.get("color", "rgb")
    out = {
        "camera": m.get("camera"),
        "ambient": (scene.get("ambientSpace") or {}).get("type", "euclidean"),
        "response": m.get("response", "radiance"),
        "maxBounces": m.get("maxBounces"),
        "maxNullCrossings": m.get("maxNullCrossings", DEFAULT_MAX_NULL_CROSSINGS),
        "scattering": m.get("scattering", "full"),
        "shadows": m.get("shadows", "opaque-dielectrics"),
        "color": color,
        "sensor": m.get("sensor", DEFAULT_SENSORS.get(color)),
    }
    if color == "spectral":
        from .spectral import MODEL_VERSION
        out["colorModelVersion"] = MODEL_VERSION
    if m.get("aovs"):
        out["aovs"] = list(m["aovs"])
    return out


def build_env_importance(table):
    """The environment importance table of the reference (src/components/env/importance.ts:16):
    Rec. 709 luminance per texel (float32 store), a 3x3 tent blur that wraps in u and clamps
    in v (float32 store), then per row the sin(theta)-weighted conditional CDF and over rows
    the marginal CDF, accumulated in float64 in index order and stored as float32.
    Returns (conditional H x W, marginal H, total weight)."""
    H, W = table.shape[:2]
    t = table.astype(np.float64)
    Y = (0.2126 * t[:, :, 0] + 0.7152 * t[:, :, 1] + 0.0722 * t[:, :, 2]).astype(np.float32)
    Yd = Y.astype(np.float64)
    acc = np.zeros((H, W), np.float64)
    for dj in (-1, 0, 1):
        rows = np.clip(np.arange(H) + dj, 0, H - 1)
        for di in (-1, 0, 1):
            cols = (np.arange(W) + di + W) % W
            w = (2 if dj == 0 else 1) * (2 if di == 0 else 1)
            acc = acc + w * Yd[rows][:, cols]
    Y = (acc / 16.0).astype(np.float32)
    sin_t = np.sin(np.pi * (np.arange(H) + 0.5) / H)
    wY = np.maximum(0.0, Y.astype(np.float64)) * sin_t[:, None]
    csum = np.cumsum(wY, axis=1)                   # sequential, like the reference's loop
    row_sum = csum[:, -1].copy()
    with np.errstate(invalid="ignore", divide="ignore"):
        cond = np.where(row_sum[:, None] > 0, csum / row_sum[:, None], 0.0).astype(np.float32)
    total = float(np.cumsum(row_sum)[-1]) if H else 0.0
    macc = np.cumsum(row_sum)
    marg = (macc / total if total > 0 else np.zeros(H)).astype(np.float32)
    return np.ascontiguousarray(cond), np.ascontiguousarray(marg), total


def _instance_spheres(placements, proto):
    """World centres and radii of a sphere batch's instances, in placement order: the
    placement record maps world -> rigid frame, so world = rotate(conj(q), s * c - t_rigid)
    (float64, then float32 like the device's placement records)."""
    pl = np.asarray(placements, np.float32).reshape(-1, 8).astype(np.float64)
    q, t, sc = pl[:, 0:4], pl[:, 4:7], pl[:, 7]
    c = np.asarray(proto[:3], np.float32).astype(np.float64)
    v = sc[:, None] * c[None, :] - t
    cq = -q[:, :3]
    c1 = np.cross(cq, v) + q[:, 3:4] * v
    c2 = np.cross(cq, c1)
    cen = (v + 2.0 * c2).astype(np.float32)
    rad = (sc * float(np.float32(proto[3]))).astype(np.float32)
    return cen, rad


def _light_bounds(rec, meshes):
    """The tree-leaf box of a light row (light descriptors' treeBounds)."""
    p = np.asarray(list(rec.p), np.float64)
    if rec.kind == abi.LIGHT_QUAD:
        pts = np.array([p[0:3], p[0:3] + p[3:6], p[0:3] + p[6:9], p[0:3] + p[3:6] + p[6:9]])
        return np.concatenate([pts.min(0), pts.max(0)])
    if rec.kind == abi.LIGHT_SPHERE:
        return np.concatenate([p[0:3] - p[3], p[0:3] + p[3]])
    if rec.kind == abi.LIGHT_MESH:
        m = meshes[int(p[0])]
        v = np.asarray(m["positions"], np.float32).reshape(-1, 3)[np.asarray(m["indices"], np.int64)]
        v = v.reshape(-1, 3).astype(np.float64)
        return np.concatenate([v.min(0), v.max(0)])
    return np.concatenate([p[0:3], p[0:3]])


def _light_tree(recs, powers, meshes):
    """Nodes and trails of the light tree over the roster (ptr_build_light_tree)."""
    from . import _native
    n = len(recs)
    boxes = np.ascontiguousarray(np.stack([_light_bounds(r, meshes) for r in recs]), np.float64)
    pw = np.ascontiguousarray(powers, np.float64)
    nodes = np.zeros(8 * (2 * n - 1), np.float32)
    trails = np.zeros(2 * n, np.uint32)
    rc = _native.load().ptr_build_light_tree(boxes.ctypes.data, pw.ctypes.data, n, nodes.ctypes.data, trails.ctypes.data)
    if rc < 0:
        raise CompileError([Diagnostic("error", "light-tree", f"light tree build failed over {n} lights")])
    return nodes, trails


def _mesh_area(positions, indices):
    """World surface area of a triangle mesh in float64 from its float32 vertices
    (lights/mesh/mesh.ts:52-62 meshWorldArea; mesh objects carry world positions)."""
    p = np.asarray(positions, np.float32).reshape(-1, 3).astype(np.float64)
    t = np.asarray(indices, np.int64).reshape(-1, 3)
    u = p[t[:, 1]] - p[t[:, 0]]
    v = p[t[:, 2]] - p[t[:, 0]]
    c = np.cross(u, v)
    a = np.sqrt(c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1] + c[:, 2] * c[:, 2]) / 2.0
    return float(np.cumsum(a)[-1]) if len(a) else 0.0   # the sequential float64 sum


def _light_power(kind, e, geom):
    """Emitted power for the selection CDF, from the authored float64 values like the
    kind descriptors (lights/quad/quad.ts:46 pi*A*Le, sphere.ts:24 pi*4*pi*r^2*Le,
    point.ts:24 4*pi*I, mesh.ts:34-36 pi*A_total*Le; radiantScalar = channel mean)."""
    mean = (e[0] + e[1] + e[2]) / 3.0
    if kind in (abi.LIGHT_QUAD, abi.LIGHT_MESH):   # lights/mesh/mesh.ts:34-36: pi*A_total*Le
        return max(1e-8, math.pi * geom * mean)
    if kind == abi.LIGHT_SPHERE:
        return max(1e-8, math.pi * 4 * math.pi * geom * geom * mean)
    return max(1e-8, 4 * math.pi * mean)


def _qrot(q, v):
    """Rotate v by unit quaternion q = (x, y, z, w): v + 2 q.xyz x (q.xyz x v + w v)."""
    qv = q[:3]
    c1 = _cross(qv, v)
    t = [c1[i] + q[3] * v[i] for i in range(3)]
    c2 = _cross(qv, t)
    return [v[i] + 2.0 * c2[i] for i in range(3)]


def _as_bytes(recs, ctype):
    n = len(recs)
    arr = (ctype * max(n, 1))()
    for i, r in enumerate(recs):
        arr[i] = r
    buf = np.frombuffer(bytes(arr), dtype=np.uint8).reshape(max(n, 1), -1)[:n].copy()
    return buf
