"""The oracle's spectral walk on the CPU against exact expected values (float64 quadrature).

The oracle restates the reference's spectral colour model (color/spectral/spectral.glsl:1-10
wavelengths_sample and :27-33 color_to_pixel, lookup.glsl:38-59 over the same lifted
ptr_spectrum records the device reads, blackbody.glsl:4-10, sensor/cie1931/cie1931.glsl:3-5).
Before it serves as the device's per-sample checker it is pinned here to the model's
definition: a pixel's film value is int S(lambda) L(lambda) dlambda over the sampled range.
Gates: the image mean within 4 standard errors and 1 % of the quadrature; a grey scene's
spectral image equals the RGB walk times the sensor's white within 4 standard errors.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.spectral import SpectralModel, LAMBDA_MIN, LAMBDA_MAX

CAM = {"camera.position": [0, 0, 3], "camera.target": [0, 0, -1], "camera.fov": 0.2}


def _strategy(max_bounces=4, lo=LAMBDA_MIN, hi=LAMBDA_MAX, wavelengths="visible", direct="none"):
    return {"id": "spectral", "measurement": {"camera": {"type": "pinhole", "fov": 0.2}, "maxBounces": max_bounces,
                                              "color": "spectral", "wavelengthRange": [lo, hi]},
            "estimator": {"directLighting": direct, "russianRoulette": None, "wavelengths": wavelengths}}


def _render(oracle_lib, scene, st, W, H, spp, params):
    r, pk = Compiler().compile(scene, st)
    o = oracle_lib.render(pk, r, W, H, spp, salt=3, params=params)
    return o["mean"], o["var"]


def _check(img, var, spp, expect):
    m = img.reshape(-1, 3).mean(axis=0)
    se = np.sqrt(var.reshape(-1, 3).mean(axis=0) / (spp * img.shape[0] * img.shape[1]))
    assert np.all(np.abs(m - expect) <= 4 * se + 0.01 * np.abs(expect) + 1e-6), (m, expect, se)


def _quad(model, f, lo=LAMBDA_MIN, hi=LAMBDA_MAX, n=200001):
    lam = np.linspace(lo, hi, n)
    return np.trapezoid(f(lam)[:, None] * model.sensor(lam), lam, axis=0)


def _panel(emission):
    return {"id": "panel", "objects": [
        {"type": "quad", "parameters": {"corner": [-5, -5, -1], "edge1": [10, 0, 0], "edge2": [0, 10, 0]},
         "material": "panel"}],
        "materials": {"panel": {"model": "lambert", "albedo": [0, 0, 0], "emission": emission, "sampleAsLight": False}},
        "lights": []}


@pytest.mark.parametrize("kind,lo,hi", [("visible", LAMBDA_MIN, LAMBDA_MAX), ("uniform", 380.0, 780.0),
                                        ("visible", 380.0, 780.0)])
def test_oracle_blackbody_panel(oracle_lib, kind, lo, hi):
    model = SpectralModel.bundled()
    img, var = _render(oracle_lib, _panel({"blackbody": {"kelvin": 3000.0, "scale": 2.0}}),
                       _strategy(lo=lo, hi=hi, wavelengths=kind), 16, 16, 128, CAM)
    spec = model.blackbody(3000.0, 2.0)
    _check(img, var, 128, _quad(model, lambda lam: model.eval(spec, lam), lo, hi))


def test_oracle_chromatic_emission_and_beer_lambert(oracle_lib):
    model = SpectralModel.bundled()
    rgb = [1.0, 0.8, 0.6]
    img, var = _render(oracle_lib, _panel(rgb), _strategy(), 16, 16, 128, CAM)
    _check(img, var, 128, _quad(model, lambda lam: model.eval(model.emission(rgb), lam)))
    sa = [0.5, 1.0, 2.0]
    scene = _panel([1.0, 1.0, 1.0])
    scene["objects"].append({"type": "box", "parameters": {"center": [0, 0, 0.5], "halfSize": [4, 4, 0.25]},
                             "material": "ink"})
    scene["materials"]["ink"] = {"model": "none", "medium": {"sigma_a": sa, "sigma_s": [0, 0, 0]}}
    img, var = _render(oracle_lib, scene, _strategy(), 16, 16, 256, CAM)
    coef, white = model.coefficient(sa), model.emission([1.0, 1.0, 1.0])
    _check(img, var, 256, _quad(model, lambda lam: model.eval(white, lam) * np.exp(-model.eval(coef, lam) * 0.5)))


def test_oracle_spectral_furnace(oracle_lib):
    model = SpectralModel.bundled()
    scene = {"id": "furnace", "objects": [{"type": "sphere", "parameters": {"center": [0, 0, 0], "radius": 1.0},
                                           "material": "grey"}],
             "materials": {"grey": {"model": "lambert", "albedo": [0.8, 0.8, 0.8]}}, "lights": [],
             "environment": {"type": "constant", "color": [1.0, 1.0, 1.0], "intensity": 1.0}}
    img, var = _render(oracle_lib, scene, _strategy(max_bounces=8), 16, 16, 256,
                       {"camera.position": [0, 0, 3.5], "camera.target": [0, 0, 0], "camera.fov": 0.1})
    sky = _quad(model, lambda lam: model.eval(model.emission([1.0, 1.0, 1.0]), lam))
    _check(img, var, 256, 0.8 * sky)


def test_oracle_grey_cornell_spectral_equals_rgb(oracle_lib):
    sc, st = scenes.cornell(direct="mis")
    sc = dict(sc, materials={k: (dict(v, albedo=[0.6, 0.6, 0.6]) if "albedo" in v else v)
                             for k, v in sc["materials"].items()})
    W = H = 32
    spp = 128
    cam = {"camera.position": [0, 1, 4], "camera.target": [0, 1, 0], "camera.fov": 0.698}
    rgb_img, rgb_var = _render(oracle_lib, sc, st, W, H, spp, cam)
    st_s = dict(st, measurement=dict(st["measurement"], color="spectral"))
    sp_img, sp_var = _render(oracle_lib, sc, st_s, W, H, spp, cam)
    model = SpectralModel.bundled()
    white = _quad(model, lambda lam: model.eval(model.emission([1.0, 1.0, 1.0]), lam))
    a = rgb_img.reshape(-1, 3).mean(axis=0) * white
    b = sp_img.reshape(-1, 3).mean(axis=0)
    se = np.sqrt((rgb_var.reshape(-1, 3).mean(axis=0) + sp_var.reshape(-1, 3).mean(axis=0)) / (spp * W * H))
    assert np.all(np.abs(a - b) <= 4 * se + 2e-3 * np.abs(a)), (a, b, se)


def test_oracle_renders_the_media_spectral_workload(oracle_lib):
    """The media + spectral configuration (chromatic medium in an IOR-1.33 boundary, a grey
    null-interface medium, a 3000 K sphere light under equiangular sampling and a quad) on
    the oracle: finite, and its RGB twin's image agrees with the spectral one in luminance
    order of magnitude (the two measure different spectra, so only the scale is checked)."""
    sc, st, _ = scenes.media_scene()
    r, pk = Compiler().compile(sc, st)
    o = oracle_lib.render(pk, r, 24, 24, 8, salt=1)
    assert np.isfinite(o["mean"]).all() and o["mean"].mean() > 0.0
