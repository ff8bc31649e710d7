"""Mesh area lights (lights/mesh/mesh.glsl:18-75, lights/mesh/mesh.ts:20-95).

An emissive Lambert material on a mesh object makes the object a one-sided light: the
triangle is picked from the normalised cumulative world-area CDF, a uniform point on it by
the square-root map, and the density d^2 / (A_total cos_l) does not depend on which
triangle was hit.  These CPU tests pin the compiler's light record, the authored-record
rejection, and the estimator on the oracle:

* the quad-panel witness: the Cornell ceiling panel as four fanned triangles of unequal
  area renders the image of the authored quad light;
* estimator equality for a 320-triangle icosphere emitter: BSDF sampling alone, NEE and MIS
  converge to the same image (MIS weights of light-sampled and BSDF-sampled paths sum to
  one only when the emitter-hit density matches the sampler's);
* a zero-area triangle first in the CDF is never picked (the strictly-greater search).
The CUDA path is compared with the oracle sample by sample in the GPU parity tests.
"""
import math

import numpy as np
import pytest

from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200.compiler import CompileError, Compiler


def _light(pk, i):
    rec = abi.Light.from_buffer_copy(bytes(pk.lights[i]))
    return rec


def test_compiler_makes_a_mesh_light():
    sc, st = scenes.cornell_mesh_light(emitter="panel")
    r, pk = Compiler().compile(sc, st)
    assert len(pk.lights) == 1
    l = _light(pk, 0)
    assert l.kind == abi.LIGHT_MESH
    region = len(sc["objects"]) - 1
    assert l.region == region
    assert int(l.p[0]) == 0 and l.p[0] == 0.0          # the scene's only mesh
    assert l.p[12] == pytest.approx(0.25, rel=1e-6)   # world area of the 0.5 x 0.5 panel
    assert l.select_pdf == pytest.approx(1.0) and l.select_cdf == pytest.approx(1.0)
    assert tuple(l.radiance)[:3] == (15.0, 15.0, 15.0)


def test_mesh_light_power_joins_the_selection_cdf():
    """pi * A_total * Le beside the quad's pi * A * Le (mesh.ts:34-36)."""
    sc, st = scenes.cornell_mesh_light(emitter="panel")
    sc = dict(sc, lights=[{"kind": "quad", "corner": [-0.9, 1.99, -0.9], "edge1": [0.5, 0, 0],
                           "edge2": [0, 0, 0.25], "emission": 10.0}])
    _, pk = Compiler().compile(sc, st)
    kinds = [_light(pk, i).kind for i in range(len(pk.lights))]
    assert kinds == [abi.LIGHT_QUAD, abi.LIGHT_MESH]
    p_quad = math.pi * 0.125 * 10.0
    p_mesh = math.pi * 0.25 * 15.0
    assert _light(pk, 1).select_pdf == pytest.approx(p_mesh / (p_quad + p_mesh), rel=1e-6)


def test_mesh_light_routes_and_rejections():
    sc, st = scenes.cornell_mesh_light(emitter="panel")
    # sampleAsLight false: the object still emits on hits but is no light
    off = dict(sc, materials=dict(sc["materials"], lamp=dict(sc["materials"]["lamp"], sampleAsLight=False)))
    _, pk = Compiler().compile(off, st)
    assert len(pk.lights) == 0
    # authored mesh light records are rejected with the route to take instead
    bad = dict(sc, lights=[{"kind": "mesh", "emission": 1.0}])
    with pytest.raises(CompileError, match="emissive material used by a mesh object"):
        Compiler().compile(bad, st)


def _render(oracle_lib, sc, st, w, h, spp, salt=3):
    r, pk = Compiler().compile(sc, st)
    return oracle_lib.render(pk, r, w, h, spp, salt=salt)


def _blocks(img, b):
    h, w, c = img.shape
    return img[: h - h % b, : w - w % b].reshape(h // b, b, w // b, b, c).mean(axis=(1, 3))


def _agree(a, b, spp, block=8, z=4.0):
    """Block means of two independent renders within z standard errors."""
    ma, mb = _blocks(a["mean"], block), _blocks(b["mean"], block)
    va = _blocks(a["var"], block) / (spp * block * block)
    vb = _blocks(b["var"], block) / (spp * block * block)
    se = np.sqrt(va + vb) + 1e-9
    zs = np.abs(ma - mb) / se
    return zs


def test_panel_mesh_light_equals_quad_light(oracle_lib):
    for direct in ("nee", "mis"):
        q = _render(oracle_lib, *scenes.cornell(direct=direct), 48, 48, 128)
        m = _render(oracle_lib, *scenes.cornell_mesh_light(direct=direct, emitter="panel"), 48, 48, 128, salt=4)
        zs = _agree(q, m, 128)
        assert zs.max() < 4.5, (direct, zs.max())
        assert (zs < 3.0).mean() > 0.97, (direct, (zs < 3.0).mean())
        tot = abs(q["mean"].mean() - m["mean"].mean())
        se = math.sqrt((q["var"].mean() + m["var"].mean()) / (128 * 48 * 48))
        assert tot < 4.0 * se, (direct, tot, se)


def test_icosphere_emitter_estimators_agree(oracle_lib):
    """BSDF-only, NEE and MIS renders of the icosphere-lit box agree: the emitter-hit
    density (hit's winding normal, total area) matches the sampler's."""
    spp = {"none": 512, "nee": 128, "mis": 128}
    out = {d: _render(oracle_lib, *scenes.cornell_mesh_light(direct=d, emitter="sphere"), 32, 32, spp[d], salt=7)
           for d in spp}
    for a, b in (("none", "nee"), ("nee", "mis"), ("none", "mis")):
        ma, mb = out[a]["mean"].mean(), out[b]["mean"].mean()
        se = math.sqrt(out[a]["var"].mean() / (spp[a] * 1024) + out[b]["var"].mean() / (spp[b] * 1024))
        assert abs(ma - mb) < 4.0 * se, (a, b, ma, mb, se)
        zs = _agree(out[a], out[b], min(spp[a], spp[b]))
        assert (zs < 3.0).mean() > 0.9, (a, b, zs)


def _degenerate_panel(direct):
    sc, st = scenes.cornell_mesh_light(direct=direct, emitter="panel")
    obj = dict(sc["objects"][-1])
    # a zero-area triangle first (repeated vertex): cdf[0] = 0 never exceeds a draw
    obj["indices"] = [[1, 1, 2]] + list(obj["indices"])
    sc = dict(sc, objects=list(sc["objects"][:-1]) + [obj])
    return sc, st


def test_zero_area_triangle_is_never_sampled(oracle_lib):
    sc, st = _degenerate_panel("nee")
    d = _render(oracle_lib, sc, st, 32, 32, 64)
    assert np.isfinite(d["sum"]).all()
    p = _render(oracle_lib, *scenes.cornell_mesh_light(direct="nee", emitter="panel"), 32, 32, 64)
    # the CDF's first entry is 0, every other entry equal: the same triangles for the same draws
    np.testing.assert_allclose(d["mean"], p["mean"], rtol=1e-5, atol=1e-6)
