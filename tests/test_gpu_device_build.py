"""Mesh BVHs built on the device (ptr_set_accel_build(PTR_BUILD_DEVICE)) on the GPU.

The device builder (a linear BVH over Morton codes, its preorder binary layout and a
greedy eight-wide collapse into the same quantized 80-byte nodes) replaces the host's SAH
builders at upload.  Every box it writes must contain its triangles, so the walks return
the exact nearest hit; with the walks' tie rule the hit IDs are those of a brute-force
scan bit for bit, and a render's samples equal the host-built scene's sample for sample.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import CudaEngine
from test_gpu_mesh import _plain_mesh_scene, _rays, _trace

pytestmark = pytest.mark.gpu


@pytest.fixture
def dev_engine():
    eng = CudaEngine(0)
    eng.set_accel_build("device")
    yield eng
    eng.close()


@pytest.mark.parametrize("level,n_rays", [(5, 20000), (8, 5000)])
def test_device_built_mesh_hits_equal_brute_force(dev_engine, oracle_lib, level, n_rays):
    sc, st = _plain_mesh_scene(level)
    r, pk = Compiler().compile(sc, st)
    dev_engine.register_scene(pk)
    rays = _rays(n_rays, 1)
    bprim, bt = oracle_lib.mesh_brute(pk, 0, rays)
    assert (bprim >= 0).sum() > n_rays // 4
    for accel in (abi.ACCEL_BVH, abi.ACCEL_CWBVH):
        reg, el, prim, t = _trace(dev_engine, accel, rays)
        np.testing.assert_array_equal(prim, bprim)
        np.testing.assert_array_equal(t[bprim >= 0], bt[bprim >= 0])


@pytest.mark.parametrize("n_tris", [1, 2, 3, 4, 9, 1000])
def test_device_build_of_small_meshes(dev_engine, oracle_lib, n_tris):
    """Meshes of one to a few triangles (a leaf root; roots of only leaf children) and a
    small random soup, against brute force."""
    rng = np.random.RandomState(n_tris)
    v = rng.uniform(-1, 1, (3 * n_tris, 3)).astype(np.float32)
    f = np.arange(3 * n_tris, dtype=np.uint32).reshape(-1, 3)
    sc = {"id": "soup", "objects": [{"kind": "mesh", "positions": v.reshape(-1), "indices": f.reshape(-1), "material": "m"}],
          "materials": {"m": {"model": "lambert"}}, "lights": []}
    st = {"id": "s", "measurement": {"camera": {}, "maxBounces": 2},
          "estimator": {"directLighting": "none", "russianRoulette": None}}
    r, pk = Compiler().compile(sc, st)
    dev_engine.register_scene(pk)
    rays = _rays(4000, 2, spread=0.8, dist=3.0)
    bprim, bt = oracle_lib.mesh_brute(pk, 0, rays)
    assert (bprim >= 0).any()
    for accel in (abi.ACCEL_BVH, abi.ACCEL_CWBVH):
        reg, el, prim, t = _trace(dev_engine, accel, rays)
        np.testing.assert_array_equal(prim, bprim)
        np.testing.assert_array_equal(t[bprim >= 0], bt[bprim >= 0])


def test_device_built_instances_equal_the_oracle(dev_engine, oracle_lib):
    sc, st, _ = scenes.mesh_scene(level=4, instances=9, env_size=(64, 32))
    r, pk = Compiler().compile(sc, st)
    dev_engine.register_scene(pk)
    rays = _rays(40000, 2, spread=3.0, dist=10.0)
    oreg, oel, oprim, ot = oracle_lib.trace_closest(pk, r, rays)
    for accel in (abi.ACCEL_BVH, abi.ACCEL_CWBVH):
        reg, el, prim, t = _trace(dev_engine, accel, rays)
        np.testing.assert_array_equal(reg, oreg)
        np.testing.assert_array_equal(prim, oprim)
        np.testing.assert_array_equal(el[oprim >= 0], oel[oprim >= 0])
        np.testing.assert_array_equal(t[oreg >= 0], ot[oreg >= 0])


@pytest.mark.parametrize("accel", ["bvh", "cwbvh"])
def test_device_built_scene_renders_the_host_built_samples(dev_engine, engine, accel):
    """The mesh workload (instanced noisy icosphere, GGX with per-triangle alpha, image
    sky): the same samples from a device-built and a host-built upload."""
    sc, st, _ = scenes.mesh_scene(level=5, instances=6, env_size=(128, 64), accel=accel)
    r, pk = Compiler().compile(sc, st)
    out = []
    for eng in (engine, dev_engine):
        eng.register_scene(pk)
        eng.load_renderer(r)
        eng.select_renderer(r.id)
        eng.params = {}
        eng.pin_reset_salt(4)
        eng.reset()
        out.append(eng.render_samples(64, 36, 4))
    np.testing.assert_array_equal(out[1], out[0])
