"""Tiled production renders on the GPU (TiledRenderer, src/app/TiledRenderer.ts:63-143).

CudaEngine.render_tiled renders each tile through ptr_frame.pixel_offset and
ptr_frame.image_size from a fresh accumulation under one pinned salt.  The stitched
picture must equal the full-frame render of the same salt (each pixel folds the same
samples in the same order), and the first tile must equal the oracle's tile sample for
sample under the parity gates of test_gpu_parity.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import plan_tiles

pytestmark = pytest.mark.gpu


def test_tiled_render_equals_the_full_frame(engine):
    sc, st = scenes.cornell(direct="mis")
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    engine.params = {}
    W, H, spp = 160, 120, 8
    engine.pin_reset_salt(21)
    engine.render_frame(W, H, spp)
    full = engine.read_export("radiance").copy()
    full_var = engine.read_export("variance").copy()
    images, stamps = engine.render_tiled(W, H, spp, tile_size=64, pictures=("radiance", "variance"),
                                         scene_id=sc["id"])
    assert len(plan_tiles(W, H, 64)["tiles"]) == 6
    np.testing.assert_allclose(images["radiance"], full, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(images["variance"], full_var, rtol=1e-5, atol=1e-7)
    s = stamps["radiance"]
    assert s["resolution"] == [W, H] and s["spp"] == spp and s["resetSalt"] == 21
    assert s["measurement"]["maxBounces"] == st["measurement"]["maxBounces"]
    assert s["git"] and s["scene"] == sc["id"]


def test_tile_matches_the_oracle_tile(engine, oracle_lib):
    """A tile off the image's corner against the oracle's same tile, sample for sample."""
    import ctypes as C
    from pathtracerglsl_b200 import abi
    sc, st = scenes.cornell(direct="mis")
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    engine.params = {}
    W, H, spp, salt = 256, 256, 8, 13
    tx, ty, tw, th = 64, 128, 64, 48
    engine.pin_reset_salt(salt)
    fr = engine._frame(tw, th, spp, accumulate=False, image=(W, H))
    fr.pixel_offset = (C.c_int32 * 2)(tx, ty)
    out = np.zeros((spp, th, tw, 3), np.float32)
    rc = engine.lib.ptr_render_samples(engine.programs[engine.current], engine.scene, C.byref(fr),
                                       out.ctypes.data_as(C.POINTER(C.c_float)), out.size)
    assert rc == abi.PTR_OK
    o = oracle_lib.render(pk, r, tw, th, spp, salt=salt, keep_samples=True, pixel_offset=(tx, ty), image_size=(W, H))
    close = np.abs(out - o["samples"]) <= 1e-4 * np.maximum(1.0, np.abs(o["samples"]))
    assert close.all(axis=-1).mean() >= 0.999
