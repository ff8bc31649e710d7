"""Per-scene kernels (ptr_specialize): NVRTC-compiled closest-hit, shading and shadow kernels
for one scene x strategy must leave every sample bit-identical to the generic kernels.

The reference's own form of this is its Generate stage, which emits GLSL per scene x
strategy (src/compiler/generate/Generator.ts:10-91); its witness is that the generated
program renders the scene.  Here the generic library is the witness: the specialised build
folds away absent occupants and unrolls the region list, and must not change a single
sample.
"""
import numpy as np
import pytest

import ref_scenes
from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler

pytestmark = pytest.mark.gpu

CASES = {
    "cornell-mis": (lambda: scenes.cornell(direct="mis"), {}, (48, 40, 4)),
    "cornell-nee": (lambda: scenes.cornell(direct="nee"), {}, (48, 40, 4)),
    "mesh-instances": (lambda: scenes.mesh_scene(level=3, instances=6, env_size=(64, 32))[:2], {}, (48, 36, 4)),
    "cornell-rough": (lambda: scenes.cornell_rough(direct="mis"), {}, (48, 40, 4)),
    "cornell-mesh-light": (lambda: scenes.cornell_mesh_light(direct="mis", emitter="sphere"), {}, (48, 40, 4)),
    "many-lights-tree": (lambda: scenes.many_lights(direct="mis", selection="bvh"), {}, (48, 40, 4)),
    "het-blobs": (lambda: scenes.het_fog(direct="mis", kind="blobs"), {}, (40, 40, 4)),
    "fog-area-mis": (lambda: (ref_scenes.FOG_AREA, ref_scenes.FOG_AREA_MIS),
                     {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.8}, (40, 30, 4)),
    "media-spectral": (lambda: scenes.media_scene()[:2], {}, (40, 40, 4)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_specialised_kernels_leave_samples_identical(engine, case):
    make, cam, (w, h, spp) = CASES[case]
    sc, st = make()
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    engine.params = dict(cam)
    engine.pin_reset_salt(5)
    engine.reset()
    generic = engine.render_samples(w, h, spp)
    engine.specialize()
    engine.reset()
    special = engine.render_samples(w, h, spp)
    np.testing.assert_array_equal(special, generic)
    # graph-launched frames too (render_frame captures a graph per wave shape)
    engine.reset()
    engine.render_frame(w, h, spp)
    a = engine.read_export("radiance").copy()
    engine.specialize(False)
    engine.reset()
    engine.render_frame(w, h, spp)
    np.testing.assert_array_equal(engine.read_export("radiance"), a)


def test_specialisation_is_cached_and_scene_bound(engine):
    sc, st = scenes.cornell(direct="mis")
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    first = engine.specialize()
    again = engine.specialize()
    assert again == 0.0 and first >= 0.0
    engine.pin_reset_salt(2)
    engine.reset()
    ref = engine.render_samples(32, 24, 2)
    # a different scene on the same renderer falls back to the generic kernels
    sc2, st2 = scenes.cornell(direct="mis")
    sc2 = dict(sc2, objects=list(sc2["objects"][:-1]))
    _, pk2 = Compiler().compile(sc2, st2)
    engine.register_scene(pk2)
    engine.reset()
    other = engine.render_samples(32, 24, 2)
    assert not np.array_equal(other, ref)
    engine.register_scene(pk)
    engine.reset()
    np.testing.assert_array_equal(engine.render_samples(32, 24, 2), ref)


def test_specialised_replay_matches_generic_gradients(engine):
    """ptr_backward of a specialised program runs the replay (ADJ) kernels compiled for the
    same census: the forward walk is bit-identical and every gradient equals the generic
    kernels' up to the order of the float64 atomic sums."""
    from pathtracerglsl_b200 import adjoint
    sc, st, (w, h, _, _) = scenes.adjoint_scene(0, n_spheres=8, width=48, height=48)
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    engine.params = {}
    rng = np.random.RandomState(4)
    dl = rng.uniform(-1.0, 1.0, (h, w, 3)).astype(np.float32)
    engine.specialize(False)
    g_generic = engine.backward(dl, w, h, 4, salt=9)
    engine.pin_reset_salt(9)
    engine.reset()
    f_generic = engine.render_samples(w, h, 4)
    engine.specialize()
    g_special = engine.backward(dl, w, h, 4, salt=9)
    engine.pin_reset_salt(9)
    engine.reset()
    np.testing.assert_array_equal(engine.render_samples(w, h, 4), f_generic)
    live = adjoint.live_mask(pk)
    assert np.abs(g_generic[live]).max() > 0.0
    scale = np.abs(g_generic).max()
    np.testing.assert_allclose(g_special, g_generic, rtol=1e-9, atol=1e-12 * scale)
    engine.specialize(False)
