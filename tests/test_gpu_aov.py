"""First-hit pictures (components/aov: measurement.aovs ['albedo', 'normal']) on the GPU.

Closed forms, after the reference's AOV contract: with nothing in front of the first
surface the albedo picture is the material's albedo fact clamped to [0, 1] and the normal
picture the shading normal faced toward the camera, both exactly; behind a homogeneous
absorbing slab both carry the camera-ray transmittance exp(-sigma_a L); a miss is 0.  The
radiance picture of an AOV program equals the one without AOVs sample for sample.
"""
import copy
import math

import numpy as np
import pytest

import ref_scenes
from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler

pytestmark = pytest.mark.gpu


def _render(engine, sc, st, w, h, spp, params):
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    engine.params = dict(params)
    engine.pin_reset_salt(3)
    engine.reset()
    engine.render_frame(w, h, spp)
    return {k: engine.read_export(k).copy() for k in r.export_targets}


def test_cornell_aovs_closed_forms(engine):
    sc, st = scenes.cornell(direct="mis")
    st = dict(st, measurement=dict(st["measurement"], aovs=["albedo", "normal"]))
    cam = {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.8}
    out = _render(engine, sc, st, 64, 64, 4, cam)
    # the back wall above the image centre (below the ceiling light): white Lambert 0.75,
    # normal +z toward the camera
    a = out["albedo"][36:40, 30:34]
    n = out["normal"][36:40, 30:34]
    np.testing.assert_allclose(a, 0.75, atol=1e-6)
    np.testing.assert_allclose(n[..., 2], 1.0, atol=1e-5)
    np.testing.assert_allclose(n[..., :2], 0.0, atol=1e-5)
    # the glass sphere: the dielectric's albedo fact is its transmittance (1); the ceiling
    # light's material has albedo 0
    assert np.isclose(out["albedo"], 1.0, atol=1e-6).all(axis=-1).any()
    assert (out["albedo"] == 0.0).all(axis=-1).any()
    # radiance is the AOV-free program's
    plain = _render(engine, *scenes.cornell(direct="mis"), 64, 64, 4, cam)
    np.testing.assert_array_equal(out["radiance"], plain["radiance"])


def test_aovs_carry_the_camera_ray_transmittance(engine):
    """Behind the unit-thick absorbing slab (sigma_a (1, 2, 4)) a screen of albedo 0.5: the
    albedo picture is 0.5 exp(-sigma_a L), L the near-normal path length through the slab."""
    sc = copy.deepcopy(ref_scenes.SLAB)
    sc["materials"]["screen"] = dict(sc["materials"]["screen"], albedo=[0.5, 0.5, 0.5])
    st = copy.deepcopy(ref_scenes.SLAB_STRATEGY)
    st["measurement"]["aovs"] = ["albedo", "normal"]
    cam = {"camera.position": [0, 0, 8], "camera.target": [0, 0, 0], "camera.fov": 0.6}
    out = _render(engine, sc, st, 8, 8, 16, cam)
    c = out["albedo"][3:5, 3:5].reshape(-1, 3)
    # the centre pixels' rays are 2-3 degrees off the axis: L = 1 / cos = 1.001-1.002
    np.testing.assert_allclose(c, np.broadcast_to(0.5 * np.exp(-np.array([1.0, 2.0, 4.0])), c.shape), rtol=1.2e-2)
    nz = out["normal"][3:5, 3:5, 2].reshape(-1)
    np.testing.assert_allclose(nz, np.exp(-np.array([1.0, 2.0, 4.0])).mean(), rtol=1.2e-2)


def test_render_stamp(engine):
    """The reproducibility stamp (App.ts buildRenderStamp) of the frame just rendered."""
    sc, st = scenes.cornell(direct="mis")
    st = dict(st, measurement=dict(st["measurement"], aovs=["albedo"]))
    _render(engine, sc, st, 32, 24, 8, {})
    stamp = engine.render_stamp("albedo", sc["id"])
    assert stamp["picture"] == "albedo" and stamp["scene"] == "cornell-c1"
    assert stamp["spp"] == 8 and stamp["resolution"] == [32, 24] and stamp["resetSalt"] == 3
    assert stamp["strategy"]["measurement"]["aovs"] == ["albedo"] and stamp["abi"] >= 3
    # the resolved measurement (plan/measurement.ts:14-35) and the source revision
    m = stamp["measurement"]
    assert m["aovs"] == ["albedo"] and m["color"] == "rgb" and m["sensor"] == "ideal"
    assert m["maxNullCrossings"] == 32 and m["scattering"] == "full" and m["response"] == "radiance"
    assert isinstance(stamp["git"], str) and stamp["git"]
