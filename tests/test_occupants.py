"""The occupant registries: one device header plus one registry line per material model or
light kind, and one host row (the reference's occupant model, README.md:7,
src/components/materials/index.ts and src/components/lights/index.ts).

CPU checks: the device registries (csrc/device/materials/registry.cuh,
csrc/device/lights/registry.cuh) and the host rows (pathtracerglsl_b200/occupants.py) list
the same occupants with the same ids and headers; every PTR_MAT_* / PTR_LIGHT_* constant of
the C ABI has an occupant; the dispatch helpers fold a census that lacks occupants (NVRTC
compile of static assertions, no GPU).
"""
import ctypes as C
import os
import re

import pytest

from pathtracerglsl_b200 import abi, occupants

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAT_DIR = os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device", "materials")


def _device_registry():
    src = open(os.path.join(MAT_DIR, "registry.cuh")).read()
    listed = re.search(r"using MaterialModels = OccupantList<([^>]*)>;", src).group(1)
    structs = [s.strip() for s in listed.split(",") if s.strip()]
    includes = re.findall(r'#include "materials/(\w+\.cuh)"', src)
    # struct name -> (header, PTR_MAT_* name)
    found = {}
    for h in includes:
        text = open(os.path.join(MAT_DIR, h)).read()
        for name, mat in re.findall(r"struct (\w+) : MaterialModel \{\s*static constexpr int kId = (PTR_MAT_\w+);", text):
            found[name] = (h, mat)
    return structs, found


def test_device_and_host_registries_agree():
    structs, found = _device_registry()
    assert len(structs) == len(set(structs)) == len(occupants.MATERIAL_MODELS)
    dev = {}
    for s in structs:
        assert s in found, f"{s} is listed but no included header defines it"
        header, mat = found[s]
        dev[getattr(abi, mat[len("PTR_"):])] = header
    host = {m.model: m.header for m in occupants.MATERIAL_MODELS.values()}
    assert dev == host


def test_device_and_host_light_registries_agree():
    d = os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device", "lights")
    src = open(os.path.join(d, "registry.cuh")).read()
    listed = [x.strip() for x in re.search(r"using LightKinds = OccupantList<([^>]*)>;", src).group(1).split(",") if x.strip()]
    found = {}
    for h in re.findall(r'#include "lights/(\w+\.cuh)"', src):
        text = open(os.path.join(d, h)).read()
        for name, kind in re.findall(r"struct (\w+) : LightKind \{\s*static constexpr int kId = (PTR_LIGHT_\w+);", text):
            found[name] = (h, kind)
    assert len(listed) == len(set(listed)) == len(occupants.LIGHT_KIND_ROWS)
    dev = {getattr(abi, found[x][1][len("PTR_"):]): found[x][0] for x in listed}
    assert dev == {k.kind: k.header for k in occupants.LIGHT_KIND_ROWS.values()}
    text = open(os.path.join(ROOT, "include", "ptx_rt.h")).read()
    assert {int(v) for v in re.findall(r"#define PTR_LIGHT_[A-Z_]+ (\d+)", text)} == set(occupants.LIGHT_BY_ID)


def test_every_abi_material_constant_has_a_model():
    text = open(os.path.join(ROOT, "include", "ptx_rt.h")).read()
    ids = {int(v) for v in re.findall(r"#define PTR_MAT_[A-Z_]+ (\d+)", text)}
    assert ids == set(occupants.MATERIAL_BY_ID)


def test_host_rows_drive_packing_and_adjoint_masks():
    """The compiler packs the model id of the row and the IOR row of models that have one;
    the adjoint's live slots follow the rows."""
    from pathtracerglsl_b200 import adjoint, scenes
    from pathtracerglsl_b200.compiler import Compiler
    sc, st, _ = scenes.adjoint_scene(0, n_spheres=12)
    _, pk = Compiler().compile(sc, st)
    mats = adjoint._materials(pk)
    regs = adjoint._regions(pk)
    mask = adjoint.live_mask(pk)
    used = {r.material for r in regs}
    for i, m in enumerate(mats):
        row = occupants.MATERIAL_BY_ID[m.model]
        live_color = bool(row.grad_color) and not (m.flags & abi.MATF_EMISSIVE) and not (row.grad_ior and i not in used)
        assert mask[i, abi.GRAD_COLOR_R] == live_color
        assert mask[i, abi.GRAD_ALPHA] == (row.grad_alpha and live_color)
    for r in regs:
        if r.material >= 0 and not occupants.MATERIAL_BY_ID[mats[r.material].model].ior:
            assert r.ior == 1.0


def _nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"):
        try:
            return C.CDLL(name)
        except OSError:
            continue
    pytest.skip("NVRTC not available")


FOLD_CHECKS = b"""
typedef signed char int8_t; typedef unsigned char uint8_t; typedef short int16_t;
typedef unsigned short uint16_t; typedef int int32_t; typedef unsigned int uint32_t;
typedef long long int64_t; typedef unsigned long long uint64_t;
#include "wavefront.cuh"
using namespace ptx;
// a Lambert + dielectric census: the other models are absent
static_assert(MatPresent<Lambert>::value && MatPresent<Dielectric>::value, "present");
static_assert(!MatPresent<GGX>::value && !MatPresent<RoughDielectric>::value, "absent");
static_assert(MatNonDelta<Lambert>::value && !MatNonDelta<Dielectric>::value, "non-delta filter");
static_assert(any_of<MatNonDelta>(MaterialModels{}), "Lambert is non-delta");
static_assert(!any_of<MatNonDelta>(OccupantList<Dielectric, GGX, Mirror, Null, RoughDielectric>{}), "no other non-delta model");
static_assert(!any_of<LightPresent>(OccupantList<SphereLight, PointLight, MeshLight>{}) && LightPresent<QuadLight>::value,
              "a quad-light census");
__global__ void probe(int model, float* out) {
    float v = 0.0f;
    auto f = [&](auto M) { v = (float)decltype(M)::kId + 1.0f; };
    dispatch_material<MatNonDelta, true>(model, f);
    out[0] = v;
}
"""


def test_dispatch_folds_absent_models():
    lib = _nvrtc()
    opts = [b"-arch=sm_100a", b"-std=c++17", b"-fmad=false", b"-default-device",
            ("-I" + os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device")).encode(),
            ("-I" + os.path.join(ROOT, "include")).encode(),
            f"-DPTR_SPEC_MATS={(1 << abi.MAT_LAMBERT) | (1 << abi.MAT_DIELECTRIC)}u".encode(),
            f"-DPTR_SPEC_LIGHTS={1 << abi.LIGHT_QUAD}u".encode()]
    prog = C.c_void_p()
    assert lib.nvrtcCreateProgram(C.byref(prog), FOLD_CHECKS, b"fold.cu", 0, None, None) == 0
    try:
        arr = (C.c_char_p * len(opts))(*opts)
        rc = lib.nvrtcCompileProgram(prog, len(opts), arr)
        size = C.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, C.byref(size))
        log = C.create_string_buffer(size.value)
        lib.nvrtcGetProgramLog(prog, log)
        assert rc == 0, log.value.decode(errors="replace")[:4000]
    finally:
        lib.nvrtcDestroyProgram(C.byref(prog))
