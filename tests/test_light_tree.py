"""Light-tree selection (estimator.lightSelection 'bvh'): accel/light_tree/light_tree.ts,
light_tree.glsl and the walk pair of compiler/generate/features/lighting.ts:767-940.

CPU checks of the builder (ptr_build_light_tree) and the estimator on the oracle:

* the reference's builder invariants (light_tree.ts vitests): exactly 2n - 1 nodes, one
  light per leaf, every trail lands on its own leaf, subtree powers add up, parents' boxes
  hold their children's, depth within the 48-level cap, coincident lights handled;
* the selection pmf sums to one over all lights for queries without a normal and for
  two-sided queries (no culling), and to at most one with a one-sided normal (a culled
  box contributes zero, variance only);
* compiler rules: instanced emitters become tree lights only under 'bvh' with NEE, the
  environment takes 1/2 of the selection, equiangular and driven emission are rejected;
* estimator equality on the oracle: 'bvh' and 'power' selection converge to the same
  image (surfaces, and a scattering medium whose events query without a normal).
The CUDA path is compared with the oracle sample by sample in the GPU tests.
"""
import math

import numpy as np
import pytest

from pathtracerglsl_b200 import _native, abi, scenes
from pathtracerglsl_b200.compiler import CompileError, Compiler

CAM = {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0]}


def _build(boxes, powers):
    boxes = np.ascontiguousarray(boxes, np.float64)
    powers = np.ascontiguousarray(powers, np.float64)
    n = len(powers)
    nodes = np.zeros(8 * (2 * n - 1), np.float32)
    trails = np.zeros(2 * n, np.uint32)
    depth = _native.load().ptr_build_light_tree(boxes.ctypes.data, powers.ctypes.data, n, nodes.ctypes.data,
                                                trails.ctypes.data)
    return depth, nodes.reshape(-1, 8), trails.reshape(-1, 2)


def _importance(bmin, bmax, phi, p, n, two_sided):
    """float64 twin of the device importance (light_tree.glsl:28-77)."""
    c = 0.5 * (bmin + bmax)
    e = bmax - bmin
    d = c - p
    d2 = d @ d
    base = phi / max(d2, max(0.25 * (e @ e), 1e-8))
    if n @ n < 0.5:
        return base
    far = np.where(n >= 0.0, bmax, bmin)
    h = n @ (far - p)
    if two_sided:
        h = max(h, -(n @ (bmin + bmax - far - p)))
    elif h <= 0.0:
        return 0.0
    cos_c = (n @ d) / math.sqrt(max(d2, 1e-12))
    if two_sided:
        cos_c = abs(cos_c)
    dmx = np.maximum(p - bmin, bmax - p)
    lo = h / math.sqrt(max(dmx @ dmx, 1e-12))
    return base * min(1.0, max(cos_c, lo))


def _pmf(nodes, trails, light, p, n, two_sided=False):
    tw, ni, pmf = int(trails[light, 0]), 0, 1.0
    for lvl in range(48):
        link = nodes[ni, 7]
        if link < 0:
            assert int(-link - 1) == light
            return pmf
        if lvl == 24:
            tw = int(trails[light, 1])
        L, R = ni + 1, int(link)
        il = _importance(nodes[L, 0:3].astype(np.float64), nodes[L, 4:7].astype(np.float64), float(nodes[L, 3]), p, n, two_sided)
        ir = _importance(nodes[R, 0:3].astype(np.float64), nodes[R, 4:7].astype(np.float64), float(nodes[R, 3]), p, n, two_sided)
        if il + ir <= 0.0:
            return 0.0
        pl = il / (il + ir)
        if tw & 1:
            pmf *= 1.0 - pl
            ni = R
        else:
            pmf *= pl
            ni = L
        tw >>= 1
    raise AssertionError("trail longer than 48 levels")


def _random_lights(n, seed, coincident=0):
    rng = np.random.RandomState(seed)
    c = rng.uniform(-5, 5, (n, 3))
    if coincident:
        c[:coincident] = c[0]
    r = rng.uniform(0.0, 0.3, (n, 1))
    r[rng.rand(n) < 0.2] = 0.0        # point lights: degenerate boxes
    boxes = np.concatenate([c - r, c + r], axis=1)
    powers = rng.lognormal(0.0, 1.5, n)
    return boxes, powers


@pytest.mark.parametrize("n,coincident", [(1, 0), (2, 0), (7, 0), (300, 0), (300, 120), (4096, 0)])
def test_builder_invariants(n, coincident):
    boxes, powers = _random_lights(n, n + coincident, coincident)
    depth, nodes, trails = _build(boxes, powers)
    assert 0 <= depth <= 47
    assert len(nodes) == 2 * n - 1
    leaves = sorted(int(-x - 1) for x in nodes[:, 7] if x < 0)
    assert leaves == list(range(n))
    for i in range(len(nodes)):
        link = nodes[i, 7]
        if link < 0:
            li = int(-link - 1)
            np.testing.assert_allclose(nodes[i, 3], powers[li], rtol=1e-6)
            np.testing.assert_allclose(nodes[i, 0:3], boxes[li, 0:3].astype(np.float32))
            continue
        L, R = i + 1, int(link)
        assert i + 1 < R < len(nodes)
        np.testing.assert_allclose(nodes[i, 3], nodes[L, 3] + nodes[R, 3], rtol=1e-5)
        assert (nodes[i, 0:3] <= np.minimum(nodes[L, 0:3], nodes[R, 0:3])).all()
        assert (nodes[i, 4:7] >= np.maximum(nodes[L, 4:7], nodes[R, 4:7])).all()
    # every trail replays onto its own leaf (asserted inside _pmf)
    p = np.array([0.3, -0.2, 0.1])
    for l in range(n):
        _pmf(nodes, trails, l, p, np.zeros(3))


def test_builder_rejects_bad_input():
    boxes, powers = _random_lights(4, 1)
    bad = powers.copy()
    bad[2] = 0.0
    assert _build(boxes, bad)[0] == abi.PTR_E_INVALID
    nanbox = boxes.copy()
    nanbox[1, 3] = np.nan
    assert _build(nanbox, powers)[0] == abi.PTR_E_INVALID


@pytest.mark.parametrize("n", [5, 64, 500])
def test_pmf_sums_to_one(n):
    boxes, powers = _random_lights(n, 7 * n)
    _, nodes, trails = _build(boxes, powers)
    rng = np.random.RandomState(n)
    for _ in range(6):
        p = rng.uniform(-6, 6, 3)
        nrm = rng.normal(size=3)
        nrm /= np.linalg.norm(nrm)
        free = sum(_pmf(nodes, trails, l, p, np.zeros(3)) for l in range(n))
        assert abs(free - 1.0) < 1e-9
        two = sum(_pmf(nodes, trails, l, p, nrm, True) for l in range(n))
        assert abs(two - 1.0) < 1e-9
        one = sum(_pmf(nodes, trails, l, p, nrm) for l in range(n))
        assert one <= 1.0 + 1e-9
        # a one-sided query never selects a light box wholly below its horizon
        for l in range(n):
            far = np.where(nrm >= 0.0, boxes[l, 3:6], boxes[l, 0:3])
            if nrm @ (far - p) < -1e-6:
                assert _pmf(nodes, trails, l, p, nrm) == 0.0


def test_compiler_tree_roster_and_rules():
    sc, st = scenes.many_lights(selection="bvh", n=16)
    r, pk = Compiler().compile(sc, st)
    assert r.program.light_tree == 1
    assert len(pk.lights) == 2 + 16                 # quad + mesh panel, then the 16 lamps
    assert [b.get("light_base", -1) for b in pk.batches] == [2, 10]
    lamp = abi.Light.from_buffer_copy(bytes(pk.lights[2]))
    assert lamp.kind == abi.LIGHT_SPHERE and lamp.region == -1
    pl = sc["objects"][7]["placements"][0]
    np.testing.assert_allclose(list(lamp.p)[:3], pl["position"], atol=1e-6)
    assert lamp.p[3] == pytest.approx(pl["scale"], rel=1e-6)
    assert len(pk.light_tree) == 8 * (2 * 18 - 1) and len(pk.light_trails) == 2 * 18
    # under 'power' the lamps stay path-found
    _, pk2 = Compiler().compile(*scenes.many_lights(selection="power", n=16))
    assert len(pk2.lights) == 2 and pk2.light_tree is None
    # NEE off: no tree
    r3, pk3 = Compiler().compile(*scenes.many_lights(direct="none", selection="bvh", n=16))
    assert r3.program.light_tree == 0 and pk3.light_tree is None
    # the environment takes half of the selection (lighting.ts:476-481)
    env_sc = dict(sc, environment={"type": "constant", "color": [0.2, 0.2, 0.2], "sampleAsLight": True})
    _, pk4 = Compiler().compile(env_sc, st)
    assert pk4.env["select_prob"] == 0.5
    # equiangular and driven emission keep the CDF (Validator.ts:629-665)
    eq = dict(st, estimator=dict(st["estimator"], mediumLightSampling="equiangular"))
    with pytest.raises(CompileError, match="reserved"):
        Compiler().compile(sc, eq)
    drv = dict(sc, materials=dict(sc["materials"], panel=dict(sc["materials"]["panel"], emission={"param": "e", "default": 1.0})))
    with pytest.raises(CompileError, match="constant light emission"):
        Compiler().compile(drv, st)


def _img(oracle_lib, sc, st, w, h, spp, salt):
    r, pk = Compiler().compile(sc, st)
    return oracle_lib.render(pk, r, w, h, spp, salt=salt, params=CAM)


@pytest.mark.parametrize("direct,fog", [("nee", False), ("mis", False), ("mis", True)])
def test_tree_and_power_selection_agree(oracle_lib, direct, fog):
    spp = 128
    a = _img(oracle_lib, *scenes.many_lights(direct=direct, selection="bvh", fog=fog), 40, 40, spp, 3)
    b = _img(oracle_lib, *scenes.many_lights(direct=direct, selection="power", fog=fog), 40, 40, spp, 4)
    ma, mb = a["mean"].mean(), b["mean"].mean()
    se = math.sqrt(a["var"].mean() / (spp * 1600) + b["var"].mean() / (spp * 1600))
    assert abs(ma - mb) < 4.0 * se, (ma, mb, se)
    bl = lambda im: im.reshape(5, 8, 5, 8, 3).mean(axis=(1, 3))
    z = np.abs(bl(a["mean"]) - bl(b["mean"])) / (np.sqrt((bl(a["var"]) + bl(b["var"])) / (spp * 64)) + 1e-9)
    assert (z < 3.0).mean() > 0.9, z.max()
    # the tree is the lower-variance selection over many small lamps
    assert a["var"].mean() < b["var"].mean()
