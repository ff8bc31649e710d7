"""ptr_render_noalloc: the allocation-free entry point, against ptr_render.

For callers that cannot allocate device memory (they own the GPU's memory through their
own pool, or run inside a loop where an allocation is not allowed), ptr_render_noalloc
renders from the library's fixed internal array into film buffers the caller passes.
Its output must equal the regular entry point's on the same inputs: same kernels, same
counter-based samples, so the films agree to float64 rounding.  Two calls in a row are
checked (the second accumulates onto the first), because every call reuses the same
array and must start from cleared counters.
"""
import ctypes as C

import numpy as np
import pytest

from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200._native import load
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import CudaEngine

pytestmark = pytest.mark.gpu

W, H, SPP, SALT = 64, 48, 4, 5


def _frame(renderer, first, accumulate):
    fr = abi.Frame()
    fr.width, fr.height, fr.spp = W, H, SPP
    fr.first_sample = first
    fr.reset_salt = SALT
    fr.accumulate = accumulate
    fr.camera = renderer.camera({}, W, H)
    return fr


def test_noalloc_matches_render_two_calls():
    torch = pytest.importorskip("torch")
    lib = load()
    sc, st = scenes.cornell()
    renderer, packed = Compiler().compile(sc, st)

    # the regular entry point: samples 0..3, then 4..7 accumulated
    eng = CudaEngine(0)
    try:
        eng.register_scene(packed)
        eng.load_renderer(renderer)
        eng.pin_reset_salt(SALT)
        eng.render_frame(W, H, SPP)
        ref1 = eng.read_export("radiance").astype(np.float64)
        eng.render_frame(W, H, SPP)
        ref2 = eng.read_export("radiance").astype(np.float64)
    finally:
        eng.close()

    torch.cuda.set_device(0)
    sum_ = torch.zeros(H * W * 3, dtype=torch.float64, device="cuda")
    sumsq = torch.zeros(H * W * 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    desc = packed.desc()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]

    fr = _frame(renderer, 0, 0)
    rc = lib.ptr_render_noalloc(C.byref(desc), C.byref(renderer.program), C.byref(fr),
                                sum_.data_ptr(), sumsq.data_ptr(), stream)
    assert rc == abi.PTR_OK
    torch.cuda.synchronize()
    mean1 = (sum_ / SPP).cpu().numpy().reshape(H, W, 3)
    np.testing.assert_allclose(mean1, ref1, rtol=1e-6, atol=1e-7)

    fr = _frame(renderer, SPP, 1)
    rc = lib.ptr_render_noalloc(C.byref(desc), C.byref(renderer.program), C.byref(fr),
                                sum_.data_ptr(), sumsq.data_ptr(), stream)
    assert rc == abi.PTR_OK
    torch.cuda.synchronize()
    mean2 = (sum_ / (2 * SPP)).cpu().numpy().reshape(H, W, 3)
    np.testing.assert_allclose(mean2, ref2, rtol=1e-6, atol=1e-7)
    assert torch.cuda.mem_get_info()[0] == free_before   # no device memory was taken


def test_noalloc_rejects_tables_beyond_the_maximum():
    lib = load()
    sc, st = scenes.cornell()
    many = [{"type": "sphere", "parameters": {"center": [0, 0, float(i)], "radius": 0.1}, "material": "white"}
            for i in range(300)]
    renderer, packed = Compiler().compile(dict(sc, objects=sc["objects"] + many), st)
    desc = packed.desc()
    fr = _frame(renderer, 0, 0)
    dummy = C.c_double()
    rc = lib.ptr_render_noalloc(C.byref(desc), C.byref(renderer.program), C.byref(fr),
                                C.addressof(dummy), C.addressof(dummy), None)
    assert rc == abi.PTR_E_INVALID
