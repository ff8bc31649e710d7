"""The instance accel of instanced batches: the CWBVH TLAS (instanceAccel 'cwbvh', the
reference's wide instance accel, intersection/index.ts:99-158) against the binary TLAS
('tlas').  The reference's own witness is image equality of the two (Δmean 0.00 %, rmse
0.00 %, docs/fable-accel-cwbvh.md:10-12); both walks return the nearest hit, so every
sample must agree (exact ties between instances, if any, may pick another instance).
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200.compiler import Compiler

pytestmark = pytest.mark.gpu


def _sphere_cloud(n=400, seed=3):
    """A cloud of instanced spheres (params tier) in the Cornell box, like the reference's
    perf-cloud scene."""
    sc, st = scenes.cornell(direct="mis")
    rng = np.random.RandomState(seed)
    pl = [{"position": [float(x) for x in rng.uniform([-0.9, 0.1, -0.9], [0.9, 1.8, 0.9])],
           "scale": float(rng.uniform(0.5, 1.5))} for _ in range(n)]
    sc = dict(sc, objects=list(sc["objects"][:5]) + [
        {"kind": "instanced", "prototype": {"type": "sphere", "parameters": {"center": [0, 0, 0], "radius": 0.04},
                                            "material": "matte"}, "placements": pl}])
    return sc, st


@pytest.mark.parametrize("case", ["sphere-cloud", "mesh-instances"])
def test_cwbvh_tlas_equals_binary_tlas(engine, case):
    if case == "sphere-cloud":
        sc, st = _sphere_cloud()
        cam = {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.698}
    else:
        sc, st, _ = scenes.mesh_scene(level=3, instances=6, env_size=(64, 32), accel="cwbvh")
        cam = {}
    out = []
    for ia in ("tlas", "cwbvh"):
        st_i = dict(st, estimator=dict(st["estimator"], instanceAccel=ia))
        r, pk = Compiler().compile(sc, st_i)
        assert r.program.instance_accel == (abi.ACCEL_CWBVH if ia == "cwbvh" else abi.ACCEL_BVH)
        engine.register_scene(pk)
        engine.load_renderer(r)
        engine.select_renderer(r.id)
        engine.params = dict(cam)
        engine.pin_reset_salt(4)
        out.append(engine.render_samples(48, 36, 4))
    same = np.all(out[0] == out[1], axis=-1).mean()
    assert same >= 0.999, same
    assert abs(out[0].mean() - out[1].mean()) <= 1e-3 * out[0].mean()
