"""Equiangular medium NEE (transport/techniques/equiangular/equiangular.glsl:18-57).

The reference pins its correctness by the estimator equality of the `haze` witness
(tests/witnesses/index.ts:1288-1310): vertex placement and equiangular placement converge
to the same image.  Here both placements are checked on the oracle (CPU) against an exact
single-scattering value (float64 quadrature), for the reference's delta-light form and for
this library's area-light extension (quad and sphere lights, strategy key
'equiangularAreaLights'); the CUDA path is then compared with the oracle sample by sample
on the GPU (haze witness scene and a foggy room lit by a sphere and a quad light).
"""
import numpy as np
import pytest

import ref_scenes
from pathtracerglsl_b200 import abi, scenes
from pathtracerglsl_b200.compiler import CompileError, Compiler

HAZE_CAM = {"camera.position": [0, 1.2, 5], "camera.target": [0, 1.2, -1], "camera.fov": 0.9}


def haze_strategies():
    vert = ref_scenes.HAZE_NEE
    eq = dict(vert, id="pt-nee-eq", estimator=dict(vert["estimator"], mediumLightSampling="equiangular"))
    return vert, eq


def area_fog():
    """A foggy room lit by a small sphere light and a 1x1 quad light (the light set of the
    media workload) — only the area-light extension admits equiangular here."""
    sc = {
        "id": "area-fog",
        "objects": [
            {"type": "plane", "parameters": {"normal": [0, 1, 0], "offset": 0.0}, "material": "gray"},
            {"type": "plane", "parameters": {"normal": [0, 0, 1], "offset": 3.0}, "material": "gray"},
            {"type": "sphere", "parameters": {"center": [0.6, 0.6, -0.8], "radius": 0.5}, "material": "gray"},
        ],
        "materials": {
            "gray": {"model": "lambert", "albedo": [0.6, 0.55, 0.5]},
            "fog": {"model": "none", "medium": {"sigma_a": [0.02, 0.03, 0.04], "sigma_s": [0.25, 0.3, 0.35],
                                                "phase_g": 0.5}},
        },
        "lights": [
            {"kind": "sphere", "position": [-0.8, 1.6, -0.5], "radius": 0.05, "emission": [400.0, 380.0, 350.0]},
            {"kind": "quad", "corner": [-0.5, 2.8, -1.5], "edge1": [1.0, 0.0, 0.0], "edge2": [0.0, 0.0, 1.0],
             "emission": 20.0},
        ],
        "ambientMedium": "fog",
    }
    base = {"id": "pt-nee", "measurement": {"camera": {"type": "pinhole", "fov": 0.9}, "maxBounces": 12},
            "estimator": {"directLighting": "nee", "russianRoulette": {"startDepth": 4},
                          "volumeSampling": "analytic", "accumulation": {"type": "average"}},
            "view": {"tonemap": {"type": "reinhard"}}}
    eq = dict(base, id="pt-nee-eq", estimator=dict(base["estimator"], mediumLightSampling="equiangular",
                                                   equiangularAreaLights=True))
    return sc, base, eq


def area_fog_mesh():
    """area_fog with a third light: an emissive level-1 icosphere (80 triangles, radius
    0.12) — equiangular over a mesh light draws the light point from the area CDF."""
    sc, base, eq = area_fog()
    v, f = scenes.icosphere(1)
    v = v * 0.12 + np.array([0.9, 1.7, -1.2])
    sc = dict(sc, id="area-fog-mesh",
              objects=list(sc["objects"]) + [{"kind": "mesh", "positions": v.tolist(), "indices": f.tolist(),
                                               "material": "lamp", "closed": True}],
              materials=dict(sc["materials"], lamp={"model": "lambert", "albedo": [0.0, 0.0, 0.0],
                                                    "emission": [60.0, 50.0, 40.0]}))
    return sc, base, eq


AREA_CAM = {"camera.position": [0, 1.2, 4.5], "camera.target": [0, 1.0, -1], "camera.fov": 0.9}


def test_compiler_pins_equiangular_to_delta_lights():
    sc, base, eq = area_fog()
    st = dict(eq, estimator={k: v for k, v in eq["estimator"].items() if k != "equiangularAreaLights"})
    with pytest.raises(CompileError) as e:
        Compiler().compile(sc, st)
    assert any("delta (point) lights only" in d.message for d in e.value.diagnostics)
    r, _ = Compiler().compile(sc, eq)
    assert r.program.equiangular == abi.EQUIANGULAR_AREA
    vert, heq = haze_strategies()
    r, _ = Compiler().compile(ref_scenes.HAZE, heq)
    assert r.program.equiangular == abi.EQUIANGULAR_DELTA
    bad = dict(heq, estimator=dict(heq["estimator"], directLighting="mis"))
    with pytest.raises(CompileError):
        Compiler().compile(ref_scenes.HAZE, bad)


# ---- exact single scattering -------------------------------------------------------
# A camera ray through an unbounded homogeneous medium (no surfaces), one scattering event
# (maxBounces 1): the radiance is the single-scattering integral
#   L = int_0^MAX_DIST exp(-st t) ss p_HG(wi.d) Le(y) cos_l / d^2 exp(-st (d - SHADOW_BACKOFF)) dt dA
# evaluated here by float64 quadrature.  Both placements (vertex NEE and equiangular) are
# unbiased estimators of it; the light passes the ray at a fixed distance, so both have
# finite variance (at a point light ON the ray both diverge, which is why the reference's
# image-mean equality of the haze witness needs many samples).
SA, SS, G = 0.1, 0.3, 0.3
ST = SA + SS
CAM_O = np.array([0.0, 0.0, 3.0])
CAM_D = np.array([0.0, 0.0, -1.0])
SS_CAM = {"camera.position": list(CAM_O), "camera.target": list(CAM_O + CAM_D), "camera.fov": 1e-4}


def _hg(c, g):
    return (1 - g * g) / (4 * np.pi * (1 + g * g - 2 * g * c) ** 1.5)


def _single_scatter(points, weights, normals, t_end=80.0, nt=400001):
    """Quadrature of the integral above over light points y with weights Le*dA (or I)."""
    t = np.linspace(0.0, t_end, nt)
    p = CAM_O[None] + t[:, None] * CAM_D[None]
    acc = np.zeros_like(t)
    for y, w, n in zip(points, weights, normals):
        v = y[None] - p
        d = np.linalg.norm(v, axis=1)
        wi = v / d[:, None]
        cos_l = 1.0 if n is None else np.maximum(0.0, -(wi @ n))
        acc += np.exp(-ST * t) * SS * _hg(wi @ CAM_D, G) * w * cos_l * np.exp(-ST * (d - 0.002)) / d ** 2
    return np.trapezoid(acc, t)


def _ss_scene(lights):
    return {"id": "single-scatter", "objects": [], "ambientMedium": "fog", "lights": lights,
            "materials": {"fog": {"model": "none", "medium": {"sigma_a": [SA] * 3, "sigma_s": [SS] * 3,
                                                              "phase_g": G}}}}


def _ss_strategy(placement, area=False):
    est = {"directLighting": "nee", "russianRoulette": None, "volumeSampling": "analytic",
           "mediumLightSampling": placement}
    if area:
        est["equiangularAreaLights"] = True
    return {"id": f"ss-{placement}", "measurement": {"camera": {"type": "pinhole", "fov": 1e-4}, "maxBounces": 1},
            "estimator": est}


def _check_single_scatter(oracle_lib, lights, exact, area):
    for placement in ("vertex", "equiangular"):
        r, pk = Compiler().compile(_ss_scene(lights), _ss_strategy(placement, area))
        spp = 1024
        o = oracle_lib.render(pk, r, 8, 8, spp, salt=3, params=SS_CAM)
        m = o["mean"][..., 0].mean()
        se = np.sqrt(o["var"][..., 0].sum() / spp) / 64
        assert abs(m - exact) <= 4.0 * se and abs(m - exact) <= 0.02 * exact, (placement, m, exact, se)


def test_single_scatter_point_light_exact(oracle_lib):
    """The reference's form: a delta light, position + intensity (lighting_query_delta)."""
    pos, intensity = np.array([0.0, 0.6, -1.0]), 10.0
    exact = _single_scatter([pos], [intensity], [None])
    _check_single_scatter(oracle_lib, [{"kind": "point", "position": list(pos), "emission": intensity}], exact, False)


def test_single_scatter_quad_light_exact(oracle_lib):
    """The area-light extension: a one-sided 0.5 x 0.5 quad light emitting downwards."""
    corner, e1, e2, le = np.array([-0.25, 0.8, -1.25]), np.array([0.5, 0, 0]), np.array([0, 0, 0.5]), 20.0
    n = 32
    u = (np.arange(n) + 0.5) / n
    pts = [corner + a * e1 + b * e2 for a in u for b in u]
    nrm = np.cross(e1, e2)
    area = np.linalg.norm(nrm)
    nrm = nrm / area
    exact = _single_scatter(pts, [le * area / len(pts)] * len(pts), [nrm] * len(pts), t_end=60.0, nt=12001)
    light = {"kind": "quad", "corner": list(corner), "edge1": list(e1), "edge2": list(e2), "emission": le}
    _check_single_scatter(oracle_lib, [light], exact, True)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["haze", "area", "area-mesh"])
def test_equiangular_cuda_matches_oracle(engine, oracle_lib, case):
    from test_gpu_parity import compare
    if case == "haze":
        _, st = haze_strategies()
        compare(engine, oracle_lib, ref_scenes.HAZE, st, 40, 30, 8, HAZE_CAM, salt=5)
    elif case == "area":
        sc, _, st = area_fog()
        compare(engine, oracle_lib, sc, st, 40, 30, 8, AREA_CAM, salt=5)
    else:
        sc, _, st = area_fog_mesh()
        compare(engine, oracle_lib, sc, st, 40, 30, 8, AREA_CAM, salt=5)


def test_equiangular_over_a_mesh_light_converges_to_vertex_placement(oracle_lib):
    """The haze witness's estimator equality with a mesh light among the lights: the
    equiangular placement (light point from the area CDF) and the at-vertex placement give
    the same image on the oracle."""
    sc, base, eq = area_fog_mesh()
    imgs = []
    for k, st in enumerate((base, eq)):
        r, pk = Compiler().compile(sc, st)
        assert abi.LIGHT_MESH in [abi.Light.from_buffer_copy(bytes(x)).kind for x in pk.lights]
        imgs.append(oracle_lib.render(pk, r, 24, 18, 256, salt=21 + k, params=AREA_CAM))
    a, b = imgs
    ma, mb = a["mean"].mean(), b["mean"].mean()
    se = np.sqrt(a["var"].mean() / (256 * 24 * 18) + b["var"].mean() / (256 * 24 * 18))
    assert abs(ma - mb) < 4.0 * se, (ma, mb, se)
    bl = lambda im: im[:18, :24].reshape(3, 6, 4, 6, 3).mean(axis=(1, 3))
    z = np.abs(bl(a["mean"]) - bl(b["mean"])) / (np.sqrt((bl(a["var"]) + bl(b["var"])) / (256 * 36)) + 1e-9)
    assert (z < 3.0).mean() > 0.9, z
