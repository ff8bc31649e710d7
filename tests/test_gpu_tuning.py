"""Launch tuning (ptr_set_tuning) and the autotuner: the knobs change scheduling only.

Every path's walk depends on its own counter-based random numbers only, so the occupant-
sorted shading queue, the ray-coherence queue order, the block size and the pool capacity
(waves of any size) must leave every sample bit-identical.  No counterpart in the reference.
"""
import numpy as np
import pytest

import ref_scenes
from pathtracerglsl_b200 import autotune, scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import CudaEngine, EngineError

pytestmark = pytest.mark.gpu

CASES = {
    "cornell-mis": (lambda: scenes.cornell(direct="mis"), {}),
    "fog-area-mis": (lambda: (ref_scenes.FOG_AREA, ref_scenes.FOG_AREA_MIS),
                     {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.8}),
    "media-spectral": (lambda: scenes.media_scene()[:2], {}),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_sorting_block_and_capacity_leave_samples_identical(engine, case):
    make, cam = CASES[case]
    sc, st = make()
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    engine.params = dict(cam)
    out = []
    for t in ({"capacity": 0, "block": 256, "sort_buckets": 1}, {"capacity": 0, "block": 256, "sort_buckets": 16},
              {"capacity": 4096, "block": 128, "sort_buckets": 8}, {"capacity": 0, "block": 256, "ray_sort": 1},
              {"capacity": 4096, "block": 128, "sort_buckets": 16, "ray_sort": 1}):
        engine.set_tuning(**t)
        engine.pin_reset_salt(9)
        engine.reset()
        out.append(engine.render_samples(160, 120, 8))   # 153,600 paths: above the sorts' 65,536-entry floor
    engine.set_tuning()
    for o in out[1:]:
        np.testing.assert_array_equal(o, out[0])


def test_tuning_validation_and_autotune(engine):
    with pytest.raises(EngineError):
        engine.set_tuning(block=192)
    with pytest.raises(EngineError):
        engine.set_tuning(sort_buckets=0)
    with pytest.raises(EngineError):
        engine.set_tuning(ray_sort=2)
    sc, st = scenes.cornell()
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    cands = [{"capacity": 1 << 16, "block": 256, "sort_buckets": 1}, {"capacity": 1 << 18, "block": 128, "sort_buckets": 8}]
    rec = autotune.tune(engine, lambda: engine.render_frame(64, 64, 8), cands)
    assert len(rec["results"]) == 2 and rec["best"]["ms"] > 0
    applied = engine.get_tuning()
    assert {k: rec["best"][k] for k in applied} == applied
    engine.set_tuning()
