"""ptr_render_noalloc: the allocation-free entry point, against ptr_render.

For callers that cannot allocate device memory (they own the GPU's memory through their
own pool, or run inside a loop where an allocation is not allowed), ptr_render_noalloc
renders from the library's fixed internal array into film buffers the caller passes.
Its output must equal the regular entry point's on the same inputs: same kernels, same
counter-based samples, so the films agree to float64 rounding.  Two calls in a row are
checked (the second accumulates onto the first), because every call reuses the same
array and must start from cleared counters.  Three frame shapes cover the array's path
pool (65536 paths): one wave, several waves of whole pixels, and frames with more pixels
than paths in flight (waves that split a pixel's samples).

The rejection cases run on the CPU: a malformed or unsupported scene must come back as
an error before anything reaches a device.
"""
import ctypes as C

import numpy as np
import pytest

from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200._native import load
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import CudaEngine

SALT = 5


def _frame(renderer, w, h, spp, first, accumulate):
    fr = abi.Frame()
    fr.width, fr.height, fr.spp = w, h, spp
    fr.first_sample = first
    fr.reset_salt = SALT
    fr.accumulate = accumulate
    fr.camera = renderer.camera({}, w, h)
    return fr


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,spp", [(64, 48, 4),      # one wave
                                     (64, 48, 32),     # two waves of whole pixels
                                     (320, 240, 2)])   # 76800 pixels: waves split pixels
def test_noalloc_matches_render_two_calls(w, h, spp):
    torch = pytest.importorskip("torch")
    lib = load()
    sc, st = scenes.cornell()
    renderer, packed = Compiler().compile(sc, st)

    # the regular entry point: samples 0..spp-1, then spp..2spp-1 accumulated
    eng = CudaEngine(0)
    try:
        eng.register_scene(packed)
        eng.load_renderer(renderer)
        eng.pin_reset_salt(SALT)
        eng.render_frame(w, h, spp)
        ref1 = eng.read_export("radiance").astype(np.float64)
        eng.render_frame(w, h, spp)
        ref2 = eng.read_export("radiance").astype(np.float64)
    finally:
        eng.close()

    torch.cuda.set_device(0)
    sum_ = torch.zeros(h * w * 3, dtype=torch.float64, device="cuda")
    sumsq = torch.zeros(h * w * 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    desc = packed.desc()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]

    fr = _frame(renderer, w, h, spp, 0, 0)
    rc = lib.ptr_render_noalloc(C.byref(desc), C.byref(renderer.program), C.byref(fr),
                                sum_.data_ptr(), sumsq.data_ptr(), stream)
    assert rc == abi.PTR_OK
    torch.cuda.synchronize()
    mean1 = (sum_ / spp).cpu().numpy().reshape(h, w, 3)
    np.testing.assert_allclose(mean1, ref1, rtol=1e-6, atol=1e-7)

    fr = _frame(renderer, w, h, spp, spp, 1)
    rc = lib.ptr_render_noalloc(C.byref(desc), C.byref(renderer.program), C.byref(fr),
                                sum_.data_ptr(), sumsq.data_ptr(), stream)
    assert rc == abi.PTR_OK
    torch.cuda.synchronize()
    mean2 = (sum_ / (2 * spp)).cpu().numpy().reshape(h, w, 3)
    np.testing.assert_allclose(mean2, ref2, rtol=1e-6, atol=1e-7)
    assert torch.cuda.mem_get_info()[0] == free_before   # no device memory was taken


def _call(lib, desc, renderer):
    fr = _frame(renderer, 64, 48, 4, 0, 0)
    dummy = C.c_double()
    return lib.ptr_render_noalloc(C.byref(desc), C.byref(renderer.program), C.byref(fr),
                                  C.addressof(dummy), C.addressof(dummy), None)


def test_noalloc_rejects_tables_beyond_the_maximum():
    lib = load()
    sc, st = scenes.cornell()
    many = [{"type": "sphere", "parameters": {"center": [0, 0, float(i)], "radius": 0.1}, "material": "white"}
            for i in range(300)]
    renderer, packed = Compiler().compile(dict(sc, objects=sc["objects"] + many), st)
    assert _call(lib, packed.desc(), renderer) == abi.PTR_E_INVALID


def _with_lights(desc, edit):
    """A copy of desc's light table with edit(lights) applied; returns (desc, keep-alive)."""
    n = desc.n_lights
    arr = (abi.Light * n)()
    C.memmove(arr, desc.lights, C.sizeof(abi.Light) * n)
    edit(arr)
    desc.lights = C.cast(arr, C.POINTER(abi.Light))
    return desc, arr


def _set_kind(kind):
    def edit(lights):
        lights[0].kind = kind
        lights[0].p[0] = 0.0
        lights[0].p[12] = 1.0
    return edit


def _set_pdf(lights):
    lights[0].select_pdf = 0.0


def _set_region(lights):
    lights[0].region = 999


@pytest.mark.parametrize("name,edit", [("mesh light without meshes", _set_kind(abi.LIGHT_MESH)),
                                       ("unknown light kind", _set_kind(7)),
                                       ("zero selection pdf", _set_pdf),
                                       ("light region out of range", _set_region)])
def test_noalloc_rejects_malformed_lights_before_any_launch(name, edit):
    lib = load()
    renderer, packed = Compiler().compile(*scenes.cornell())
    desc, keep = _with_lights(packed.desc(), edit)
    assert _call(lib, desc, renderer) == abi.PTR_E_INVALID, name


def test_noalloc_rejects_malformed_regions_before_any_launch():
    lib = load()
    renderer, packed = Compiler().compile(*scenes.cornell())
    desc = packed.desc()
    n = desc.n_regions
    orig = packed.desc().regions
    for field, value in (("shape", -1), ("shape", abi.SHAPE_MESH), ("material", 99)):
        arr = (abi.Region * n)()
        C.memmove(arr, orig, C.sizeof(abi.Region) * n)
        setattr(arr[0], field, value)
        desc.regions = C.cast(arr, C.POINTER(abi.Region))
        assert _call(lib, desc, renderer) == abi.PTR_E_INVALID, (field, value)
    arr = (abi.Region * n)()
    C.memmove(arr, orig, C.sizeof(abi.Region) * n)
    arr[0].p[0] = float("nan")
    desc.regions = C.cast(arr, C.POINTER(abi.Region))
    assert _call(lib, desc, renderer) == abi.PTR_E_INVALID
