"""The oracle's forward-mode reference of the adjoint (oracle.forward), on the CPU.

No counterpart in the reference (it renders only).  The forward mode carries float64
tangents d throughput / d theta and d radiance / d theta along the oracle's own float32
walk, each weight site differentiating its own formula with dual numbers, under the
adjoint's conventions (sampled directions, distances, densities, MIS weights and roulette
probabilities held fixed).  Here it is pinned three ways:

* the walk it rides is the plain render's: the primal image is bit-identical;
* for parameters that move no sampling decision (Lambert albedos; a grey medium's albedo,
  since free flight samples sigma_t only) the image is smooth in the parameter along the
  same random numbers, so central differences of the oracle itself agree to rounding;
* the dielectric IOR at normal incidence, where the refracted direction does not depend on
  the IOR, against the closed form of a glass slab, d/d eta [(1 - F) / (1 + F)].

tests/test_gpu_adjoint.py then holds the GPU adjoint to this reference on every parameter.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import abi, adjoint, scenes
from pathtracerglsl_b200.compiler import Compiler


def _box():
    sc, st = scenes.adjoint_box_scene()
    return Compiler().compile(sc, st)


def test_forward_mode_rides_the_plain_walk(oracle_lib):
    import oracle
    r, pk = _box()
    f = oracle.forward(pk, r, 10, 8, 8, salt=3)
    base = oracle.render(pk, r, 10, 8, 8, salt=3)["mean"]
    np.testing.assert_array_equal(f["mean"], base)
    assert f["jac"].shape == (8, 10, 3, abi.GRAD_SLOTS * len(pk.materials))
    # slots no material uses carry no derivative
    dead = ~adjoint.live_mask(pk).reshape(-1)
    assert not np.any(f["jac"][..., dead])


def _check_linear_parameters(r, pk, W, H, spp, salt):
    """The forward mode against central differences of the oracle for the parameters that
    move no sampling decision (no roulette): the colour slots and the medium's albedo.
    Returns the number of parameters checked."""
    import oracle
    f = oracle.forward(pk, r, W, H, spp, salt=salt)
    theta = adjoint.param_table(pk)
    dl = np.random.RandomState(1).uniform(-1, 1, (H, W, 3))
    g = np.einsum("hwc,hwck->k", dl, f["jac"]).reshape(-1, abi.GRAD_SLOTS)
    mask = adjoint.live_mask(pk)
    checked = 0
    for i, k in zip(*np.nonzero(mask)):
        if k not in (abi.GRAD_COLOR_R, abi.GRAD_COLOR_G, abi.GRAD_COLOR_B, abi.GRAD_MEDIUM_ALBEDO):
            continue
        eps = 1e-2
        tp, tm = theta.copy(), theta.copy()
        tp[i, k] += eps
        tm[i, k] -= eps
        ip = oracle.render(adjoint.with_params(pk, tp), r, W, H, spp, salt=salt)["mean"]
        im = oracle.render(adjoint.with_params(pk, tm), r, W, H, spp, salt=salt)["mean"]
        fd = float((dl * (ip - im)).sum() / (2 * eps))
        assert abs(g[i, k] - fd) <= 1e-3 * abs(fd) + 1e-6, (pk.material_names[i], abi.GRAD_NAMES[k], g[i, k], fd)
        checked += 1
    return checked


def test_forward_mode_colour_slots_on_the_adjoint_scene(oracle_lib):
    """Lambert albedo, GGX F0 and dielectric transmittance (slots 0-2) of every model the
    inverse-rendering scene holds, on a reduced copy of it (8 spheres)."""
    sc, st, _ = scenes.adjoint_scene(0, n_spheres=8)
    r, pk = Compiler().compile(sc, st)
    models = {m["model"] for m in sc["materials"].values()}
    assert {"lambert", "ggx", "dielectric"} <= models
    assert _check_linear_parameters(r, pk, 12, 12, 8, 5) == 3 * (len(sc["materials"]) - 1) + 1


def test_forward_mode_matches_oracle_differences_on_linear_parameters(oracle_lib):
    import oracle
    r, pk = _box()
    W, H, spp, salt = 12, 12, 16, 3
    f = oracle.forward(pk, r, W, H, spp, salt=salt)
    theta = adjoint.param_table(pk)
    dl = np.random.RandomState(1).uniform(-1, 1, (H, W, 3))
    g = np.einsum("hwc,hwck->k", dl, f["jac"]).reshape(-1, abi.GRAD_SLOTS)
    mask = adjoint.live_mask(pk)
    checked = 0
    for i, k in zip(*np.nonzero(mask)):
        if k not in (abi.GRAD_COLOR_R, abi.GRAD_COLOR_G, abi.GRAD_COLOR_B, abi.GRAD_MEDIUM_ALBEDO):
            continue
        eps = 1e-2
        tp, tm = theta.copy(), theta.copy()
        tp[i, k] += eps
        tm[i, k] -= eps
        ip = oracle.render(adjoint.with_params(pk, tp), r, W, H, spp, salt=salt)["mean"]
        im = oracle.render(adjoint.with_params(pk, tm), r, W, H, spp, salt=salt)["mean"]
        fd = float((dl * (ip - im)).sum() / (2 * eps))
        assert abs(g[i, k] - fd) <= 1e-3 * abs(fd) + 1e-6, (pk.material_names[i], abi.GRAD_NAMES[k], g[i, k], fd)
        checked += 1
    assert checked == 16   # 4 Lambert albedos x 3 channels + the GGX F0 x 3 + the medium's albedo


def test_forward_mode_ior_exact_at_normal_incidence(oracle_lib):
    import oracle
    scene = {
        "id": "slab-ior",
        "objects": [
            {"type": "box", "parameters": {"center": [0, 0, 0], "halfSize": [1.5, 1.5, 0.1]}, "material": "glass"},
            {"type": "quad", "parameters": {"corner": [-2, -2, -1], "edge1": [4, 0, 0], "edge2": [0, 4, 0]},
             "material": "panel"},
        ],
        "materials": {"glass": {"model": "dielectric", "ior": 1.5},
                      "panel": {"model": "lambert", "albedo": [0, 0, 0], "emission": [1.0, 1.0, 1.0],
                                "sampleAsLight": False}},
        "lights": [],
    }
    st = {"id": "pt", "measurement": {"camera": {"type": "pinhole", "fov": 1e-4}, "maxBounces": 40},
          "estimator": {"directLighting": "none", "russianRoulette": None}}
    cam = {"camera.position": [0, 0, 3], "camera.target": [0, 0, -1], "camera.fov": 1e-4}
    r, pk = Compiler().compile(scene, st)
    eta = 1.5
    F = ((eta - 1) / (eta + 1)) ** 2
    dF = 2 * (eta - 1) / (eta + 1) * 2 / (eta + 1) ** 2
    exact_i = (1 - F) / (1 + F)
    exact_d = -2 * dF / (1 + F) ** 2
    f = oracle.forward(pk, r, 8, 8, 2048, salt=9, params=cam)
    assert abs(f["mean"].mean() - exact_i) < 3e-3, (f["mean"].mean(), exact_i)
    gi = f["jac"][..., abi.GRAD_SLOTS * pk.material_names.index("glass") + abi.GRAD_IOR].mean()
    assert abs(gi - exact_d) <= 0.02 * abs(exact_d), (gi, exact_d)


def test_forward_mode_rejects_programs_outside_the_adjoint(oracle_lib):
    import oracle
    sc, st, _ = scenes.media_scene(spectral=True)
    r, pk = Compiler().compile(sc, st)
    with pytest.raises(ValueError):
        oracle.forward(pk, r, 4, 4, 1)
