"""Meshes, instanced batches and the image environment on the GPU, against the oracle.

Hit IDs: the device walks (binary SAH BVH and the compressed wide BVH, 128-bit node
loads, one-FMA quantized slabs) must return exactly the triangle and t of a brute-force
scan with the same Moller-Trumbore leaf (bit-exact: same float32 operations).
Images: per-sample agreement with the oracle as in test_gpu_parity.
"""
import ctypes as C

import numpy as np
import pytest

from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200.compiler import Compiler
from test_gpu_parity import compare

pytestmark = pytest.mark.gpu


def _plain_mesh_scene(level=5):
    v, f = scenes.icosphere(level)
    v = v * (1.0 + 0.05 * scenes.value_noise(v, 3))[:, None]
    sc = {"id": "mesh", "objects": [{"kind": "mesh", "positions": v.astype(np.float32).reshape(-1),
                                      "indices": f.astype(np.uint32).reshape(-1), "material": "m"}],
          "materials": {"m": {"model": "lambert"}}, "lights": []}
    st = {"id": "s", "measurement": {"camera": {}, "maxBounces": 2},
          "estimator": {"directLighting": "none", "russianRoulette": None}}
    return sc, st


def _rays(n, seed, spread=0.9, dist=3.0):
    rng = np.random.RandomState(seed)
    o = rng.normal(size=(n, 3))
    o = o / np.linalg.norm(o, axis=1, keepdims=True) * dist
    tgt = rng.normal(size=(n, 3)) * spread
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.ascontiguousarray(np.concatenate([o, d], 1).astype(np.float32))


def _trace(engine, accel, rays):
    n = len(rays)
    reg = np.zeros(n, np.int32)
    el = np.zeros(n, np.int32)
    prim = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    engine._check(engine.lib.ptr_trace_closest(engine.ctx, engine.scene, accel, rays.ctypes.data, n,
                                               reg.ctypes.data, el.ctypes.data, prim.ctypes.data, t.ctypes.data))
    return reg, el, prim, t


_BRUTE = {}   # (level, rays seed) -> the brute-force answer, shared by both walks


@pytest.mark.parametrize("level", [5, 8])
@pytest.mark.parametrize("accel", [abi.ACCEL_BVH, abi.ACCEL_CWBVH])
def test_mesh_hit_ids_bit_exact_vs_brute_force(engine, oracle_lib, accel, level):
    """20,000 rays against the level-5 icosphere (20,480 triangles) and the level-8 one of
    the mesh configuration (1,310,720 triangles): triangle and t equal to a brute-force
    scan, ties included (the lower triangle index wins on both sides)."""
    sc, st = _plain_mesh_scene(level)
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    rays = _rays(20000, 1)
    reg, el, prim, t = _trace(engine, accel, rays)
    if (level, 1) not in _BRUTE:
        _BRUTE[level, 1] = oracle_lib.mesh_brute(pk, 0, rays)
    bprim, bt = _BRUTE[level, 1]
    assert (bprim >= 0).sum() > 5000
    np.testing.assert_array_equal(prim, bprim)
    np.testing.assert_array_equal(t[bprim >= 0], bt[bprim >= 0])


@pytest.mark.parametrize("accel", [abi.ACCEL_BVH, abi.ACCEL_CWBVH])
@pytest.mark.parametrize("instance_accel", ["tlas", "cwbvh"])
def test_instanced_mesh_hits_match_oracle(engine, oracle_lib, accel, instance_accel):
    """Instanced meshes: region, instance, triangle and t equal to the oracle's ordered scan
    over the instances, bit for bit, whichever TLAS and BLAS the device walks."""
    sc, st, _ = scenes.mesh_scene(level=4, instances=9, env_size=(64, 32))
    st = dict(st, estimator=dict(st["estimator"], instanceAccel=instance_accel))
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    engine.load_renderer(r)
    rays = _rays(40000, 2, spread=3.0, dist=10.0)
    reg, el, prim, t = _trace(engine, accel, rays)
    oreg, oel, oprim, ot = oracle_lib.trace_closest(pk, r, rays)
    assert (oprim >= 0).sum() > 2000
    np.testing.assert_array_equal(reg, oreg)
    np.testing.assert_array_equal(prim, oprim)
    inst = oprim >= 0
    np.testing.assert_array_equal(el[inst], oel[inst])
    np.testing.assert_array_equal(t[oreg >= 0], ot[oreg >= 0])


def test_instanced_ties_resolve_to_the_lower_instance(engine, oracle_lib):
    """Two placements of one mesh at the same pose: every hit on them is a tie at equal t,
    which both sides give to the first placement (the reference scans its instances in
    order with a strict nearer-than test)."""
    v, f = scenes.icosphere(3)
    proto = {"kind": "mesh", "positions": v.astype(np.float32).reshape(-1), "indices": f.astype(np.uint32).reshape(-1),
             "material": "m"}
    place = [{"position": [0.5, 0.0, 0.0], "scale": 1.0}, {"position": [0.5, 0.0, 0.0], "scale": 1.0},
             {"position": [-1.5, 0.0, 0.0], "scale": 1.0}]
    sc = {"id": "ties", "objects": [{"kind": "instanced", "prototype": proto, "placements": place}],
          "materials": {"m": {"model": "lambert"}}, "lights": []}
    st = {"id": "s", "measurement": {"camera": {}, "maxBounces": 2},
          "estimator": {"directLighting": "none", "russianRoulette": None, "meshTraversal": "cwbvh"}}
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    rays = _rays(5000, 3, spread=1.5, dist=6.0)
    for accel in (abi.ACCEL_BVH, abi.ACCEL_CWBVH):
        reg, el, prim, t = _trace(engine, accel, rays)
        oreg, oel, oprim, ot = oracle_lib.trace_closest(pk, r, rays)
        hit = oprim >= 0
        assert hit.sum() > 500 and not (oel[hit] == 1).any()
        np.testing.assert_array_equal(reg, oreg)
        np.testing.assert_array_equal(el[hit], oel[hit])
        np.testing.assert_array_equal(prim, oprim)


@pytest.mark.parametrize("accel", ["bvh", "cwbvh"])
def test_mesh_workload_image_matches_oracle(engine, oracle_lib, accel):
    sc, st, _ = scenes.mesh_scene(level=3, instances=4, env_size=(128, 64), accel=accel)
    compare(engine, oracle_lib, sc, st, 48, 27, 8, {})


def test_image_environment_furnace(engine, oracle_lib):
    """A Lambert sphere (albedo 0.8) inside a uniform image environment of radiance 1:
    the image-env sampler, its pdf and the MIS weights must reproduce rho = 0.8."""
    sc, st = scenes.furnace()
    sc = dict(sc, environment={"type": "image", "table": np.ones((32, 64, 3), np.float32), "intensity": 1.0})
    compare(engine, oracle_lib, sc, st, 32, 32, 16, {})
    engine.reset()
    engine.render_frame(32, 32, 4096)
    c = engine.read_export("radiance")[12:20, 12:20].mean()
    assert abs(c - 0.8) < 1e-3 * 0.8, c
