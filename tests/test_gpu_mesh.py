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


@pytest.mark.parametrize("accel", [abi.ACCEL_BVH, abi.ACCEL_CWBVH])
def test_mesh_hit_ids_bit_exact_vs_brute_force(engine, oracle_lib, accel):
    sc, st = _plain_mesh_scene(5)
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    rays = _rays(20000, 1)
    reg, el, prim, t = _trace(engine, accel, rays)
    bprim, bt = oracle_lib.mesh_brute(pk, 0, rays)
    assert (bprim >= 0).sum() > 5000
    np.testing.assert_array_equal(prim, bprim)
    np.testing.assert_array_equal(t[bprim >= 0], bt[bprim >= 0])


@pytest.mark.parametrize("accel", [abi.ACCEL_BVH, abi.ACCEL_CWBVH])
def test_instanced_mesh_hits_match_oracle(engine, oracle_lib, accel):
    sc, st, _ = scenes.mesh_scene(level=4, instances=9, env_size=(64, 32))
    r, pk = Compiler().compile(sc, st)
    engine.register_scene(pk)
    rays = _rays(40000, 2, spread=3.0, dist=10.0)
    reg, el, prim, t = _trace(engine, accel, rays)
    oreg, oprim, ot = oracle_lib.trace_closest(pk, r, rays)
    mesh_hits = oprim >= 0
    assert mesh_hits.sum() > 2000
    assert (reg == oreg).mean() > 0.9999
    assert (prim == oprim).mean() > 0.9999
    np.testing.assert_allclose(t[mesh_hits & (prim == oprim)], ot[mesh_hits & (prim == oprim)], rtol=0, atol=0)


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
