"""Spectral transport on the GPU against exact expected values (float64 quadrature).

No generated program of the reference's snapshot uses the spectral colour model, so these
checks restate its expectation directly: the film value of a pixel is
  E[0.25 sum_i S(lambda_i) L(lambda_i) / p(lambda_i)] = int S(lambda) L(lambda) dlambda
over the sampled range (color/spectral/spectral.glsl:27-33), with S the CIE 1931 sensor
(sensor/cie1931/cie1931.glsl:3-5) and L the lifted spectra (lookup.glsl:38-59, blackbody.glsl).
Gates: the image mean within 4 standard errors and 1 % of the quadrature.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import CudaEngine
from pathtracerglsl_b200.spectral import SpectralModel, LAMBDA_MIN, LAMBDA_MAX

pytestmark = pytest.mark.gpu

CAM = {"camera.position": [0, 0, 3], "camera.target": [0, 0, -1], "camera.fov": 0.2}


def _render(scene, st, W, H, spp, params=None, salt=3):
    r, pk = Compiler().compile(scene, st)
    eng = CudaEngine(0)
    try:
        eng.register_scene(pk)
        eng.load_renderer(r)
        eng.params = dict(params or {})
        eng.pin_reset_salt(salt)
        eng.render_frame(W, H, spp)
        return eng.read_export("radiance").astype(np.float64), eng.read_export("variance").astype(np.float64), pk
    finally:
        eng.close()


def _strategy(max_bounces=4, lo=LAMBDA_MIN, hi=LAMBDA_MAX, wavelengths="visible", direct="none"):
    return {"id": "spectral", "measurement": {"camera": {"type": "pinhole", "fov": 0.2}, "maxBounces": max_bounces,
                                              "color": "spectral", "wavelengthRange": [lo, hi]},
            "estimator": {"directLighting": direct, "russianRoulette": None, "wavelengths": wavelengths}}


def _check(img, var, spp, expect):
    m = img.reshape(-1, 3).mean(axis=0)
    se = np.sqrt(var.reshape(-1, 3).mean(axis=0) / (spp * img.shape[0] * img.shape[1]))
    assert np.all(np.abs(m - expect) <= 4 * se + 0.01 * np.abs(expect) + 1e-6), (m, expect, se)


def _quad(model, f, lo=LAMBDA_MIN, hi=LAMBDA_MAX, n=200001):
    lam = np.linspace(lo, hi, n)
    return np.trapezoid(f(lam)[:, None] * model.sensor(lam), lam, axis=0)


def _panel(emission):
    """A camera facing an emissive quad that fills the view (one-sided, facing +z)."""
    return {"id": "panel", "objects": [
        {"type": "quad", "parameters": {"corner": [-5, -5, -1], "edge1": [10, 0, 0], "edge2": [0, 10, 0]},
         "material": "panel"}],
        "materials": {"panel": {"model": "lambert", "albedo": [0, 0, 0], "emission": emission, "sampleAsLight": False}},
        "lights": []}


@pytest.mark.parametrize("kind,lo,hi", [("visible", LAMBDA_MIN, LAMBDA_MAX), ("uniform", 380.0, 780.0),
                                        ("visible", 380.0, 780.0)])
def test_blackbody_panel(kind, lo, hi):
    model = SpectralModel.bundled()
    img, var, _ = _render(_panel({"blackbody": {"kelvin": 3000.0, "scale": 2.0}}), _strategy(lo=lo, hi=hi, wavelengths=kind),
                          16, 16, 256, CAM)
    spec = model.blackbody(3000.0, 2.0)
    _check(img, var, 256, _quad(model, lambda lam: model.eval(spec, lam), lo, hi))


def test_chromatic_emission_panel():
    model = SpectralModel.bundled()
    rgb = [1.0, 0.8, 0.6]
    img, var, _ = _render(_panel(rgb), _strategy(), 16, 16, 256, CAM)
    expect = _quad(model, lambda lam: model.eval(model.emission(rgb), lam))
    _check(img, var, 256, expect)
    assert np.all(np.abs(expect - rgb) < 1e-3)    # the lift reproduces the authored colour


def test_chromatic_beer_lambert():
    """A D65-white panel seen through an absorbing slab (null interface) whose sigma_a is
    the lifted coefficient (0.5, 1.0, 2.0): int S(l) D65(l) exp(-sigma(l) d) dl."""
    model = SpectralModel.bundled()
    sa = [0.5, 1.0, 2.0]
    scene = _panel([1.0, 1.0, 1.0])
    scene["objects"].append({"type": "box", "parameters": {"center": [0, 0, 0.5], "halfSize": [4, 4, 0.25]},
                             "material": "ink"})
    scene["materials"]["ink"] = {"model": "none", "medium": {"sigma_a": sa, "sigma_s": [0, 0, 0]}}
    img, var, _ = _render(scene, _strategy(), 16, 16, 512, CAM)
    coef = model.coefficient(sa)
    white = model.emission([1.0, 1.0, 1.0])
    expect = _quad(model, lambda lam: model.eval(white, lam) * np.exp(-model.eval(coef, lam) * 0.5))
    _check(img, var, 512, expect)


def test_spectral_furnace():
    """A grey Lambert sphere (albedo 0.8) in a constant white environment: 0.8 of the sky's
    sensor response on the sphere (every bounce off a convex sphere sees the sky)."""
    model = SpectralModel.bundled()
    scene = {"id": "furnace", "objects": [{"type": "sphere", "parameters": {"center": [0, 0, 0], "radius": 1.0},
                                           "material": "grey"}],
             "materials": {"grey": {"model": "lambert", "albedo": [0.8, 0.8, 0.8]}}, "lights": [],
             "environment": {"type": "constant", "color": [1.0, 1.0, 1.0], "intensity": 1.0}}
    img, var, _ = _render(scene, _strategy(max_bounces=8), 16, 16, 512,
                          {"camera.position": [0, 0, 3.5], "camera.target": [0, 0, 0], "camera.fov": 0.1})
    sky = _quad(model, lambda lam: model.eval(model.emission([1.0, 1.0, 1.0]), lam))
    _check(img, var, 512, 0.8 * sky)


def test_grey_cornell_spectral_equals_rgb():
    """With grey colours everywhere the spectral walk must converge to the RGB walk (the D65
    white integrates to the sensor's white): the image means agree within 4 standard errors."""
    sc, st = scenes.cornell(direct="mis")
    sc = dict(sc, materials={k: (dict(v, albedo=[0.6, 0.6, 0.6]) if "albedo" in v else v)
                             for k, v in sc["materials"].items()})
    W = H = 64
    spp = 256
    cam = {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.698}
    rgb_img, rgb_var, _ = _render(sc, st, W, H, spp, cam)
    st_s = dict(st, measurement=dict(st["measurement"], color="spectral"))
    sp_img, sp_var, _ = _render(sc, st_s, W, H, spp, cam)
    model = SpectralModel.bundled()
    white = _quad(model, lambda lam: model.eval(model.emission([1.0, 1.0, 1.0]), lam))
    a = rgb_img.reshape(-1, 3).mean(axis=0) * white
    b = sp_img.reshape(-1, 3).mean(axis=0)
    se = np.sqrt((rgb_var.reshape(-1, 3).mean(axis=0) + sp_var.reshape(-1, 3).mean(axis=0)) / (spp * W * H))
    assert np.all(np.abs(a - b) <= 4 * se + 2e-3 * np.abs(a)), (a, b, se)


def test_media_workload_renders():
    """The media + spectral workload at a small size: finite, non-negative on average, and
    the spectral program's device guards stay clear."""
    sc, st, _ = scenes.media_scene()
    r, pk = Compiler().compile(sc, st)
    eng = CudaEngine(0)
    try:
        eng.register_scene(pk)
        eng.load_renderer(r)
        eng.pin_reset_salt(1)
        eng.render_frame(48, 48, 16)
        img = eng.read_export("radiance")
        assert np.isfinite(img).all() and img.mean() > 0.0
        assert eng.counters()["error_flags"] == 0
    finally:
        eng.close()


# ---- the device against the oracle's spectral walk, sample for sample ------------------
# Same packed scene, same counter-based random numbers, same four wavelengths per sample
# (the oracle restates wavelengths_sample, the lifted-record evaluation and color_to_pixel):
# the gates of test_gpu_parity.compare.

@pytest.mark.parametrize("spectral", [True, False], ids=["spectral", "rgb"])
def test_media_workload_matches_oracle(engine, oracle_lib, spectral):
    """The media + spectral configuration itself: a chromatic medium (sigma_t 0.5, 1, 2)
    inside an IOR-1.33 boundary, a grey null-interface medium, a 3000 K sphere light under
    equiangular sampling and a quad at radiance 20, depth 64; and its RGB twin."""
    from test_gpu_parity import compare
    sc, st, _ = scenes.media_scene(spectral=spectral)
    compare(engine, oracle_lib, sc, st, 48, 48, 8, {})


@pytest.mark.parametrize("case", ["furnace", "blackbody", "grey-cornell"])
def test_spectral_witnesses_match_oracle(engine, oracle_lib, case):
    from test_gpu_parity import compare
    if case == "furnace":
        scene = {"id": "furnace", "objects": [{"type": "sphere", "parameters": {"center": [0, 0, 0], "radius": 1.0},
                                               "material": "grey"}],
                 "materials": {"grey": {"model": "lambert", "albedo": [0.8, 0.8, 0.8]}}, "lights": [],
                 "environment": {"type": "constant", "color": [1.0, 1.0, 1.0], "intensity": 1.0}}
        compare(engine, oracle_lib, scene, _strategy(max_bounces=8), 24, 24, 16,
                {"camera.position": [0, 0, 3.5], "camera.target": [0, 0, 0], "camera.fov": 0.6})
    elif case == "blackbody":
        compare(engine, oracle_lib, _panel({"blackbody": {"kelvin": 3000.0, "scale": 2.0}}),
                _strategy(lo=380.0, hi=780.0, wavelengths="uniform"), 16, 16, 16, CAM)
    else:
        sc, st = scenes.cornell(direct="mis")
        st_s = dict(st, measurement=dict(st["measurement"], color="spectral"))
        compare(engine, oracle_lib, sc, st_s, 32, 32, 8,
                {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.698})
