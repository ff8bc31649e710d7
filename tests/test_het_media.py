"""Heterogeneous media (transport/volume/delta_tracking/delta_tracking.glsl; the
expression coefficients of types.ts MediumDescription).

CPU checks, after the reference's correctness gates for the occupant:
* the expression compiler: every built-in and operator, interpreted by the oracle, equals a
  float64 numpy evaluation at random points; malformed sources and a missing majorant are
  compile errors;
* F-HET-CONST: a constant written as an expression (delta tracking) renders the image of the
  same constant medium on the analytic arm;
* F-HET-SLAB: an absorbing slab with a linear sigma_a(z) transmits exp(-integral) through
  its centre (the ratio-tracked pass-through);
* F-CLAMP: a field above its majorant renders as the majorant-clamped constant.
The CUDA path is compared with the oracle sample by sample in the GPU tests, which also
check that the upload validator refuses malformed field programs.
"""
import copy
import math

import numpy as np
import pytest

import ref_scenes
from pathtracerglsl_b200 import abi, field, scenes
from pathtracerglsl_b200.compiler import CompileError, Compiler

EXPRS = [
    ("0.5 + p.x * 2.0 - p.y / 4.0", lambda p: 0.5 + p[:, 0] * 2.0 - p[:, 1] / 4.0),
    ("exp(-1.5 * p.y) * (0.6 + 0.4 * sin(2.0 * p.x) * cos(2.0 * p.z))",
     lambda p: np.exp(-1.5 * p[:, 1]) * (0.6 + 0.4 * np.sin(2 * p[:, 0]) * np.cos(2 * p[:, 2]))),
    ("dot(p - vec3(0.1, 0.2, 0.3), p) + length(p)",
     lambda p: ((p - [0.1, 0.2, 0.3]) * p).sum(1) + np.linalg.norm(p, axis=1)),
    ("vec3(1.0, 0.5, 0.25) * sqrt(abs(p.x)) + p", lambda p: np.array([1.0, 0.5, 0.25]) * np.sqrt(np.abs(p[:, :1])) + p),
    ("clamp(p.x, -0.2, 0.3) + mix(1.0, 3.0, fract(p.y)) + smoothstep(-1.0, 1.0, p.z)",
     lambda p: np.clip(p[:, 0], -0.2, 0.3) + (1.0 * (1 - (p[:, 1] - np.floor(p[:, 1]))) + 3.0 * (p[:, 1] - np.floor(p[:, 1])))
     + (lambda t: t * t * (3 - 2 * t))(np.clip((p[:, 2] + 1.0) / 2.0, 0, 1))),
    ("min(p.x, p.y) + max(p.y, p.z) + mod(p.x * 3.0, 0.7) + step(0.1, p.z) + floor(p.y * 2.0)",
     lambda p: np.minimum(p[:, 0], p[:, 1]) + np.maximum(p[:, 1], p[:, 2]) + np.mod(p[:, 0] * 3.0, 0.7)
     + (p[:, 2] >= 0.1) + np.floor(p[:, 1] * 2.0)),
    ("pow(abs(p.x) + 0.5, 1.5) + log(2.0 + p.y) - -p.z", lambda p: (np.abs(p[:, 0]) + 0.5) ** 1.5 + np.log(2 + p[:, 1]) + p[:, 2]),
    ("u_a_gain * p.x + u_b", lambda p: 2.5 * p[:, 0] + 0.75),
]


@pytest.mark.parametrize("src,ref", EXPRS)
def test_field_programs_match_numpy(oracle_lib, src, ref):
    expr = {"kind": "glsl", "source": src, "params": [{"param": "a.gain", "default": 2.5}, {"param": "b", "default": 0.0}]}
    code = field.compile_field(expr, {"b": 0.75})
    pts = np.random.RandomState(3).uniform(-1.0, 1.0, (257, 3)).astype(np.float32)
    got = oracle_lib.field_eval(code, pts).astype(np.float64)
    want = np.asarray(ref(pts.astype(np.float64)), np.float64)
    want = np.broadcast_to(want.reshape(len(pts), -1), got.shape)
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-5)


@pytest.mark.parametrize("src,msg", [("p.w", "component"), ("sin(p.x", "expected"), ("foo(p)", "unknown name"),
                                     ("dot(p, 1.0)", "dot of a scalar"), ("vec3(p.x, p)", "vec3"),
                                     ("p.x p.y", "after the expression")])
def test_field_compiler_rejects(src, msg):
    with pytest.raises(field.FieldError, match=msg):
        field.compile_field({"kind": "glsl", "source": src}, {})


def test_medium_validation():
    sc, st = scenes.het_fog(kind="ground")
    bad = copy.deepcopy(sc)
    del bad["materials"]["fog"]["medium"]["majorant"]
    with pytest.raises(CompileError, match="majorant"):
        Compiler().compile(bad, st)
    spec = dict(st, measurement=dict(st["measurement"], color="spectral"))
    with pytest.raises(CompileError, match="RGB only"):
        Compiler().compile(sc, spec)
    r, pk = Compiler().compile(sc, st)
    m = np.frombuffer(pk.materials.tobytes(), dtype=np.uint8).reshape(len(pk.materials), -1)
    recs = [abi.Material.from_buffer_copy(bytes(row)) for row in m]
    het = [x for x in recs if x.field_s]
    assert len(het) == 1 and het[0].field_a == 0 and het[0].majorant == 2.0
    assert het[0].flags & abi.MATF_SCATTERING


def _slab(sigma_a, majorant=None):
    sc = copy.deepcopy(ref_scenes.SLAB)
    for name, m in sc["materials"].items():
        if m.get("medium"):
            m["medium"] = {"sigma_a": sigma_a}
            if majorant is not None:
                m["medium"]["majorant"] = majorant
    return sc


def _slab_extent(sc):
    for o in sc["objects"]:
        mat = sc["materials"][o["material"]]
        if mat.get("medium"):
            return o
    raise AssertionError("no medium in the slab scene")


CAM = {"camera.position": [0, 0, 8], "camera.target": [0, 0, 0], "camera.fov": 0.6}


def _centre(oracle_lib, sc, st, spp=4096):
    r, pk = Compiler().compile(sc, dict(st, estimator=dict(st["estimator"], volumeSampling="delta-tracking")))
    o = oracle_lib.render(pk, r, 8, 8, spp, params=CAM)
    return o["mean"][3:5, 3:5].mean(axis=(0, 1)), o


def test_slab_linear_absorption(oracle_lib):
    """F-HET-SLAB: sigma_a = a + b z through the slab's centre integrates to exp(-a L - b (z1^2 - z0^2) / 2)."""
    box = _slab_extent(ref_scenes.SLAB)
    c, h = box["parameters"]["center"], box["parameters"]["halfSize"]
    z0, z1 = c[2] - h[2], c[2] + h[2]
    a, b = 0.6, 0.4
    sc = _slab({"kind": "glsl", "source": f"{a} + {b} * p.z"}, majorant=a + b * max(abs(z0), abs(z1)) + 0.5)
    got, _ = _centre(oracle_lib, sc, ref_scenes.SLAB_STRATEGY)
    want = math.exp(-(a * (z1 - z0) + b * (z1 * z1 - z0 * z0) / 2.0))
    np.testing.assert_allclose(got, want, rtol=0.03)


def test_constant_expression_equals_analytic(oracle_lib):
    """F-HET-CONST on absorption, and F-CLAMP: a field above its majorant is the clamp."""
    ref, _ = _centre(oracle_lib, _slab([0.7, 0.7, 0.7]), ref_scenes.SLAB_STRATEGY)
    got, _ = _centre(oracle_lib, _slab({"kind": "glsl", "source": "0.7"}, majorant=2.0), ref_scenes.SLAB_STRATEGY)
    np.testing.assert_allclose(got, ref, rtol=0.03)
    clamp_ref, _ = _centre(oracle_lib, _slab([1.5, 1.5, 1.5]), ref_scenes.SLAB_STRATEGY)
    clamped, _ = _centre(oracle_lib, _slab({"kind": "glsl", "source": "vec3(4.0, 4.0, 4.0)"}, majorant=1.5), ref_scenes.SLAB_STRATEGY)
    np.testing.assert_allclose(clamped, clamp_ref, rtol=0.05)


def test_delta_tracking_equals_analytic_scattering(oracle_lib):
    """F-HET-CONST on a scattering fog: delta tracking of a constant expression converges to
    the analytic channel-MIS arm of the same constant medium (ratio-tracked shadows too)."""
    sc, st = scenes.het_fog(kind="ground")
    const = copy.deepcopy(sc)
    const["materials"]["fog"]["medium"]["sigma_s"] = [0.5, 0.5, 0.5]
    expr = copy.deepcopy(sc)
    expr["materials"]["fog"]["medium"]["sigma_s"] = {"kind": "glsl", "source": "0.5"}
    cam = {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0]}
    imgs = []
    for k, s in enumerate((const, expr)):
        r, pk = Compiler().compile(s, st)
        imgs.append(oracle_lib.render(pk, r, 24, 24, 256, salt=9 + k, params=cam))
    a, b = imgs
    se = math.sqrt(a["var"].mean() / (256 * 576) + b["var"].mean() / (256 * 576))
    assert abs(a["mean"].mean() - b["mean"].mean()) < 4.0 * se, (a["mean"].mean(), b["mean"].mean(), se)
    bl = lambda im: im.reshape(3, 8, 3, 8, 3).mean(axis=(1, 3))
    z = np.abs(bl(a["mean"]) - bl(b["mean"])) / (np.sqrt((bl(a["var"]) + bl(b["var"])) / (256 * 64)) + 1e-9)
    assert (z < 3.0).mean() > 0.9, z.max()
