"""Scenes uploaded from the reference's packed channels (ptr_upload_scene_rails, rail v2)
against the same scenes uploaded from the scene description (ptr_upload_scene), on the GPU.

The rail path walks the reference's own BVH and TLAS node arrays and placement records in
place; with the leaf permutations given, every hit id is the caller's, so every sample is
the description path's bit for bit.  Without them hit ids are leaf indices, which only
moves equal-t ties.  A mesh light samples its triangles by the rail's leaf-order CDF (as
the reference does), a different but equally valid order: its film agrees in distribution.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import _native, rails, scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import EngineError

pytestmark = pytest.mark.gpu


def _samples(engine, r, pk, w, h, spp, upload, salt=3):
    upload()
    engine.load_renderer(r)
    engine.select_renderer(r.id)
    engine.params = {}
    engine.pin_reset_salt(salt)
    engine.reset()
    return engine.render_samples(w, h, spp)


def _both(engine, sc, st, w, h, spp, with_orders=True):
    r, pk = Compiler().compile(sc, st)
    pr = rails.pack(pk, _native.load())
    a = _samples(engine, r, pk, w, h, spp, lambda: engine.register_scene(pk))
    b = _samples(engine, r, pk, w, h, spp, lambda: engine.register_scene_rails(pk, pr, with_orders=with_orders))
    assert engine.counters()["error_flags"] == 0
    return a, b


@pytest.mark.parametrize("traversal", ["cwbvh", "bvh"])
def test_instanced_mesh_from_rails_equals_description(engine, traversal):
    """Six instances of a displaced icosphere (frame-tier placements, the binary TLAS
    and, for meshTraversal 'cwbvh', the wide BLAS built on the device from the rail's
    triangles) with per-triangle alpha."""
    sc, st, _ = scenes.mesh_scene(level=3, instances=6, env_size=(32, 16), accel=traversal)
    a, b = _both(engine, sc, st, 48, 36, 4)
    np.testing.assert_array_equal(b, a)


def test_leaf_hit_ids_only_move_ties(engine):
    sc, st, _ = scenes.mesh_scene(level=3, instances=6, env_size=(32, 16))
    a, b = _both(engine, sc, st, 48, 36, 4, with_orders=False)
    same = (a == b).all(axis=-1).mean()
    assert same >= 0.99, same


@pytest.mark.parametrize("accel", ["tlas", "cwbvh"])
def test_instanced_sphere_lights_from_rails_equal_description(engine, accel):
    """Params-tier placements (the folded world centre and radius, one texel each) of two
    batches of emissive instanced spheres under light-tree selection, through the binary
    TLAS and its wide twin (the light tree and its trails come with the description)."""
    sc, st = scenes.many_lights(direct="mis", selection="bvh")
    # without the scene's emissive mesh panel, whose rail CDF is in leaf order
    sc = dict(sc, objects=[o for o in sc["objects"] if o.get("kind") != "mesh"])
    st = dict(st, estimator=dict(st["estimator"], instanceAccel=accel))
    r, pk = Compiler().compile(sc, st)
    cam = {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.8}
    pr = rails.pack(pk, _native.load())
    out = []
    for up in (lambda: engine.register_scene(pk), lambda: engine.register_scene_rails(pk, pr)):
        up()
        engine.load_renderer(r)
        engine.select_renderer(r.id)
        engine.params = dict(cam)
        engine.pin_reset_salt(7)
        engine.reset()
        out.append(engine.render_samples(40, 40, 4))
    np.testing.assert_array_equal(out[1], out[0])


def test_mesh_light_from_rails_agrees_in_distribution(engine):
    """An emissive icosphere lights the box (NEE + MIS): the rail's leaf-order CDF and the
    description's caller-order CDF pick different triangles for the same number, so the
    two films agree within 3 standard errors per pixel, not sample for sample."""
    sc, st = scenes.cornell_mesh_light(direct="mis", emitter="sphere")
    r, pk = Compiler().compile(sc, st)
    pr = rails.pack(pk, _native.load())
    spp = 64
    a = _samples(engine, r, pk, 32, 32, spp, lambda: engine.register_scene(pk)).astype(np.float64)
    b = _samples(engine, r, pk, 32, 32, spp, lambda: engine.register_scene_rails(pk, pr), salt=11).astype(np.float64)
    se = np.sqrt((a.var(axis=0, ddof=1) + b.var(axis=0, ddof=1)) / spp)
    ok = np.abs(a.mean(axis=0) - b.mean(axis=0)) <= 3.0 * se + 1e-6
    assert ok.all(axis=-1).mean() >= 0.99
    assert not np.array_equal(a, b)


def _corrupt(pr, what):
    if what == "order":
        pr.meshes[0]["tri_order"] = pr.meshes[0]["tri_order"].copy()
        pr.meshes[0]["tri_order"][1] = pr.meshes[0]["tri_order"][0]
    elif what == "node":
        q = pr.nodes.reshape(-1, 4)
        q[pr.meshes[0]["nbase"] + 1, 3] = 1e6          # the root's right child far outside
    elif what == "index":
        q = pr.indices.reshape(-1, 4)
        q[pr.meshes[0]["tbase"] + 3, 1] = pr.meshes[0]["vertex_count"]
    elif what == "tier":
        pr.batches[0]["placement_texels"] = 1
    elif what == "span":
        pr.meshes[0]["tbase"] = len(pr.indices) // 4


@pytest.mark.parametrize("what", ["order", "node", "index", "tier", "span"])
def test_malformed_rails_are_rejected(engine, what):
    """A permutation with a repeat, a node link outside the tree, a vertex id outside the
    mesh, the wrong placement tier and a region past its channel are refused before
    anything reaches the device."""
    sc, st, _ = scenes.mesh_scene(level=2, instances=3, env_size=(16, 8))
    _, pk = Compiler().compile(sc, st)
    pr = rails.pack(pk, _native.load())
    _corrupt(pr, what)
    with pytest.raises(EngineError, match="rails"):
        engine.register_scene_rails(pk, pr)
