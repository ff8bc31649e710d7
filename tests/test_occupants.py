"""The material-model registry: one device header plus one registry line per model, and one
host row (the reference's occupant model, README.md:7 and src/components/materials/index.ts).

CPU checks: the device registry (csrc/device/materials/registry.cuh) and the host registry
(pathtracerglsl_b200/occupants.py) list the same models with the same PTR_MAT_* ids and
headers; every PTR_MAT_* constant of the C ABI has a model; the dispatch helpers fold a
census that lacks models (NVRTC compile of static assertions, no GPU).
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
    listed = re.search(r"using MaterialModels = ModelList<([^>]*)>;", src).group(1)
    structs = [s.strip() for s in listed.split(",") if s.strip()]
    includes = re.findall(r'#include "materials/(\w+\.cuh)"', src)
    # struct name -> (header, PTR_MAT_* name)
    found = {}
    for h in includes:
        text = open(os.path.join(MAT_DIR, h)).read()
        for name, mat in re.findall(r"struct (\w+) : MaterialModel \{\s*static constexpr int kModel = (PTR_MAT_\w+);", text):
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
static_assert(model_present<false, Lambert>() && model_present<false, Dielectric>(), "present");
static_assert(!model_present<false, GGX>() && !model_present<false, RoughDielectric>(), "absent");
static_assert(model_present<true, Lambert>() && !model_present<true, Dielectric>(), "non-delta filter");
static_assert(any_present<true>(MaterialModels{}), "Lambert is non-delta");
static_assert(!any_present<true>(ModelList<Dielectric, GGX, Mirror, Null, RoughDielectric>{}), "no other non-delta model");
__global__ void probe(int model, float* out) {
    float v = 0.0f;
    auto f = [&](auto M) { v = (float)decltype(M)::kModel + 1.0f; };
    dispatch_model<true>(model, f, MaterialModels{});
    out[0] = v;
}
"""


def test_dispatch_folds_absent_models():
    lib = _nvrtc()
    opts = [b"-arch=sm_100a", b"-std=c++17", b"-fmad=false", b"-default-device",
            ("-I" + os.path.join(ROOT, "pathtracerglsl_b200", "csrc", "device")).encode(),
            ("-I" + os.path.join(ROOT, "include")).encode(),
            f"-DPTR_SPEC_MATS={(1 << abi.MAT_LAMBERT) | (1 << abi.MAT_DIELECTRIC)}u".encode()]
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
