"""The path-replay adjoint (ptr_backward) against finite differences and an exact value.

No counterpart in the reference (it renders only).  Gradients are checked on the loss
linearised at the primal image, sum(dL/dI * I(theta)), so the adjoint and the finite
differences estimate the same number:
  * central differences (eps = 1e-2 on values of order 0.1-2) with common random numbers
    (the same salt for theta +- eps), no roulette;
  * gate: |g_adjoint - g_fd| / |g_fd| < 2 % over the whole gradient vector (L2), and per
    parameter for the ones whose FD is well resolved;
  * the dielectric IOR against the closed form of a glass slab seen at normal incidence
    (there the refracted direction does not depend on the IOR, so the interface terms the
    adjoint differentiates are the whole derivative): I = Le (1 - F) / (1 + F).
The inverse-rendering scene itself (64 spheres + a medium sphere, 252 parameters: every
material's full set) is checked against the float64 forward mode parameter by parameter
and against central differences with eps = 1e-3 and common random numbers.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import abi, adjoint, scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import CudaEngine, EngineError

pytestmark = pytest.mark.gpu


def box_scene():
    return scenes.adjoint_box_scene()


class Rig:
    def __init__(self, scene, strategy, W, H, params=None):
        self.r, self.pk = Compiler().compile(scene, strategy)
        self.eng = CudaEngine(0)
        self.eng.register_scene(self.pk)
        self.eng.load_renderer(self.r)
        self.eng.params = dict(params or {})
        self.W, self.H = W, H
        self.theta = adjoint.param_table(self.pk)
        self.mask = adjoint.live_mask(self.pk)

    def render(self, table, spp, salt):
        self.eng.update_params(adjoint.with_params(self.pk, table))
        self.eng.pin_reset_salt(salt)
        self.eng.reset()
        self.eng.render_frame(self.W, self.H, spp)
        return self.eng.read_export("radiance").astype(np.float64)

    def backward(self, dl, spp, salt):
        self.eng.update_params(adjoint.with_params(self.pk, self.theta))
        return self.eng.backward(dl.astype(np.float32), self.W, self.H, spp, salt=salt)

    def fd(self, dl, i, k, eps, spp, salt):
        tp = self.theta.copy()
        tp[i, k] += eps
        tm = self.theta.copy()
        tm[i, k] -= eps
        return float((dl * (self.render(tp, spp, salt) - self.render(tm, spp, salt))).sum() / (2 * eps))

    def close(self):
        self.eng.close()


def test_adjoint_matches_finite_differences():
    sc, st = box_scene()
    rig = Rig(sc, st, 48, 48)
    try:
        rng = np.random.RandomState(5)
        target = rig.render(rig.theta * (1 + 0.1 * rng.uniform(-1, 1, rig.theta.shape)), 512, 101)
        primal = rig.render(rig.theta, 512, 202)
        _, dl = adjoint.l2_loss(primal, target)
        spp = 2048
        g = rig.backward(dl, spp, salt=7)
        idx = list(zip(*np.nonzero(rig.mask)))
        fd = np.array([rig.fd(dl, i, k, 1e-2, spp, 7) for i, k in idx])
        ga = np.array([g[i, k] for i, k in idx])
        rel = np.linalg.norm(ga - fd) / np.linalg.norm(fd)
        assert rel < 0.02, (rel, list(zip(idx, ga, fd)))
        # per parameter: the ones that move no vertex (albedos) resolve to 0.5 %; GGX alpha,
        # sigma_t and g move sampled directions / distances, so their FD is noisier
        for (i, k), a, f in zip(idx, ga, fd):
            if k in (abi.GRAD_ALBEDO_R, abi.GRAD_ALBEDO_G, abi.GRAD_ALBEDO_B, abi.GRAD_MEDIUM_ALBEDO) \
                    and abs(f) > 1e-4:
                assert abs(a - f) <= 0.005 * abs(f), (rig.pk.material_names[i], abi.GRAD_NAMES[k], a, f)
            else:
                assert abs(a - f) <= 0.1 * abs(f) + 0.02 * np.abs(fd).max(), (rig.pk.material_names[i], abi.GRAD_NAMES[k], a, f)
        # the gradient does not depend on how many samples came before it beyond noise,
        # and a second call reproduces the first (float64 accumulation, order-free up to rounding)
        g2 = rig.backward(dl, spp, salt=7)
        np.testing.assert_allclose(g2, g, rtol=1e-6, atol=1e-12)
    finally:
        rig.close()


def _slab():
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
    return scene, st, cam


def test_adjoint_ior_exact_at_normal_incidence():
    scene, st, cam = _slab()
    rig = Rig(scene, st, 16, 16, params=cam)
    try:
        eta = 1.5
        F = ((eta - 1) / (eta + 1)) ** 2
        dF = 2 * (eta - 1) / (eta + 1) * 2 / (eta + 1) ** 2
        exact_i = (1 - F) / (1 + F)
        exact_d = -2 * dF / (1 + F) ** 2
        img = rig.render(rig.theta, 4096, 3)
        assert abs(img.mean() - exact_i) < 3e-3, (img.mean(), exact_i)
        dl = np.full((16, 16, 3), 1.0 / (16 * 16 * 3), np.float32)     # d(mean image)
        g = rig.backward(dl, 4096, salt=9)
        gi = g[rig.pk.material_names.index("glass"), abi.GRAD_IOR]
        assert abs(gi - exact_d) <= 0.02 * abs(exact_d), (gi, exact_d)
    finally:
        rig.close()


def test_backward_rejects_chromatic_media_and_equiangular():
    sc, st = box_scene()
    sc["materials"]["fog"] = {"model": "none", "medium": {"sigma_a": [0.3, 0.2, 0.1], "sigma_s": [1.7] * 3}}
    rig = Rig(sc, st, 8, 8)
    try:
        with pytest.raises(EngineError) as e:
            rig.eng.backward(np.zeros((8, 8, 3), np.float32), 8, 8, 1)
        assert "grey" in str(e.value)
    finally:
        rig.close()


def test_update_params_equals_fresh_upload():
    sc, st = box_scene()
    rig = Rig(sc, st, 32, 24)
    try:
        t2 = rig.theta * 1.05
        a = rig.render(t2, 4, 11)
        eng2 = CudaEngine(0)
        try:
            eng2.register_scene(adjoint.with_params(rig.pk, t2))
            eng2.load_renderer(rig.r)
            eng2.pin_reset_salt(11)
            eng2.render_frame(32, 24, 4)
            np.testing.assert_array_equal(eng2.read_export("radiance"), a.astype(np.float32))
        finally:
            eng2.close()
    finally:
        rig.close()


def test_adjoint_matches_forward_mode_reference(oracle_lib):
    """The adjoint against the oracle's float64 forward mode at 64x64.

    Both differentiate the same per-sample estimator (detached sampling, MIS weights and
    roulette probabilities held fixed) along the same random numbers, so the contracted
    gradients agree to rounding, parameter by parameter — including GGX alpha, sigma_t and
    g, whose finite differences are noisy.  The forward mode differentiates the BSDF, phase,
    Fresnel and medium formulas by dual arithmetic; the adjoint uses hand-derived
    log-derivatives, so this pins those derivations.
    """
    import oracle
    sc, st = box_scene()
    W = H = 64
    spp, salt = 64, 11
    rig = Rig(sc, st, W, H)
    try:
        rng = np.random.RandomState(23)
        dl = rng.uniform(-1.0, 1.0, (H, W, 3)) / (H * W * 3)
        g = rig.backward(dl, spp, salt=salt)
        fwd = oracle.forward(rig.pk, rig.r, W, H, spp, salt=salt)
        gf = np.einsum("hwc,hwck->k", dl, fwd["jac"]).reshape(g.shape)
        idx = list(zip(*np.nonzero(rig.mask)))
        ga = np.array([g[i, k] for i, k in idx])
        gr = np.array([gf[i, k] for i, k in idx])
        rel = np.linalg.norm(ga - gr) / np.linalg.norm(gr)
        assert rel < 2e-3, (rel, list(zip(idx, ga, gr)))
        for (i, k), a, f in zip(idx, ga, gr):
            assert abs(a - f) <= 5e-3 * abs(f) + 1e-4 * np.abs(gr).max(), (rig.pk.material_names[i], abi.GRAD_NAMES[k], a, f)
    finally:
        rig.close()


def _c5_rig(W, H):
    sc, st, _ = scenes.adjoint_scene(0)
    return Rig(sc, st, W, H)


def test_adjoint_on_the_inverse_rendering_scene_matches_forward_mode(oracle_lib):
    """Every one of the scene's ~260 parameters against the oracle's float64 forward mode at
    64 x 64 (64 spp): the same estimator on the same random numbers, so they agree to
    rounding parameter by parameter."""
    import oracle
    W = H = 64
    spp, salt = 64, 13
    rig = _c5_rig(W, H)
    try:
        assert 240 <= rig.mask.sum() <= 270
        rng = np.random.RandomState(29)
        dl = rng.uniform(-1.0, 1.0, (H, W, 3)) / (H * W * 3)
        g = rig.backward(dl, spp, salt=salt)
        fwd = oracle.forward(rig.pk, rig.r, W, H, spp, salt=salt)
        gf = np.einsum("hwc,hwck->k", dl, fwd["jac"]).reshape(g.shape)
        idx = list(zip(*np.nonzero(rig.mask)))
        ga = np.array([g[i, k] for i, k in idx])
        gr = np.array([gf[i, k] for i, k in idx])
        rel = np.linalg.norm(ga - gr) / np.linalg.norm(gr)
        assert rel < 2e-3, rel
        bad = [(rig.pk.material_names[i], abi.GRAD_NAMES[k], a, f) for (i, k), a, f in zip(idx, ga, gr)
               if abs(a - f) > 5e-3 * abs(f) + 1e-4 * np.abs(gr).max()]
        assert not bad, bad[:10]
    finally:
        rig.close()


def test_adjoint_on_the_inverse_rendering_scene_matches_finite_differences():
    """Central differences (eps = 1e-3, common random numbers: the same salt and spp as the
    adjoint) of the linearised loss, for the parameters that move no sampling decision:
    every material's colour (Lambert albedo, GGX F0, dielectric transmittance) and the
    medium's albedo — 202 of the scene's 252.  For these the differences are exact, so the
    gate is 2 % over the vector and 0.5 % per parameter.  GGX alpha, sigma_t and g move
    sampled directions and distances: with common random numbers their differences are
    dominated by the samples whose decisions flip (measured on this scene, the differences
    at eps = 1e-3 and 1e-2 disagree with each other by more than their size), so they are
    checked against the float64 forward mode above, and against differences on the box
    scene, not here.  The IOR's refracted-direction term is not propagated (documented in
    the C header)."""
    W = H = 64
    spp, salt = 512, 17
    rig = _c5_rig(W, H)
    try:
        rng = np.random.RandomState(31)
        target = rig.render(rig.theta * (1 + 0.1 * rng.uniform(-1, 1, rig.theta.shape)), 256, 301)
        primal = rig.render(rig.theta, 256, 302)
        _, dl = adjoint.l2_loss(primal, target)
        g = rig.backward(dl, spp, salt=salt)
        linear = (abi.GRAD_COLOR_R, abi.GRAD_COLOR_G, abi.GRAD_COLOR_B, abi.GRAD_MEDIUM_ALBEDO)
        idx = [(i, k) for i, k in zip(*np.nonzero(rig.mask)) if k in linear]
        assert len(idx) >= 200
        fd = np.array([rig.fd(dl, i, k, 1e-3, spp, salt) for i, k in idx])
        ga = np.array([g[i, k] for i, k in idx])
        rel = np.linalg.norm(ga - fd) / np.linalg.norm(fd)
        assert rel < 0.02, rel
        bad = [(rig.pk.material_names[i], abi.GRAD_NAMES[k], a, f) for (i, k), a, f in zip(idx, ga, fd)
               if abs(a - f) > 0.005 * abs(f) + 1e-3 * np.abs(fd).max()]
        assert not bad, bad[:10]
    finally:
        rig.close()


@pytest.mark.parametrize("log_bytes, capacity", [("0", None), ("1200000", None), (None, "4096")])
def test_hit_log_bounds_and_waves_leave_gradients_unchanged(monkeypatch, log_bytes, capacity):
    """The replay reads the forward walk's logged closest hits and shadow-query results
    (visibility, media lengths) where the log holds their walk iteration and walks the scene
    again elsewhere: with no log, a log holding only the first iterations (1.2 MB: two
    iterations of the 9216-path pool at 64 bytes a path), or a pool of several waves (the log
    rewritten per wave), every gradient is the default run's up to the order of the float64
    atomic sums."""
    W = H = 48
    rig = _c5_rig(W, H)
    try:
        rng = np.random.RandomState(5)
        dl = rng.uniform(-1.0, 1.0, (H, W, 3)) / (H * W * 3)
        ref = rig.backward(dl, 4, salt=21)
        if log_bytes is not None:
            monkeypatch.setenv("PTR_HIT_LOG_BYTES", log_bytes)
        if capacity is not None:
            monkeypatch.setenv("PTR_CAPACITY", capacity)
        g = rig.backward(dl, 4, salt=21)
        assert np.abs(ref[rig.mask]).max() > 0.0
        np.testing.assert_allclose(g, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())
    finally:
        rig.close()


def test_walk_log_walks_again_queries_through_more_than_two_media(monkeypatch):
    """A shadow record holds at most two (medium, length) pairs.  Three disjoint grey-medium
    spheres stacked under the ceiling light make the floor's shadow queries cross three
    distinct media, so the forward walk marks them and the replay walks them again: the
    gradients equal those of a run with no log, and every medium's sigma_t is live."""
    sc, st = scenes.adjoint_box_scene()
    sc = dict(sc)
    objects = list(sc["objects"][:5])
    materials = dict(sc["materials"])
    for j, (y, s) in enumerate([(0.45, 1.0), (0.95, 2.0), (1.45, 3.0)]):
        materials[f"fog{j}"] = {"model": "none", "medium": {"sigma_a": [0.1 * s] * 3, "sigma_s": [0.9 * s] * 3,
                                                            "phase_g": 0.3}}
        objects.append({"type": "sphere", "parameters": {"center": [0.0, y, -0.2], "radius": 0.2},
                        "material": f"fog{j}"})
    sc["objects"] = objects
    sc["materials"] = materials
    W = H = 48
    rig = Rig(sc, st, W, H)
    try:
        rng = np.random.RandomState(37)
        dl = rng.uniform(-1.0, 1.0, (H, W, 3)) / (H * W * 3)
        ref = rig.backward(dl, 4, salt=31)
        monkeypatch.setenv("PTR_HIT_LOG_BYTES", "0")
        g = rig.backward(dl, 4, salt=31)
        np.testing.assert_allclose(ref, g, rtol=1e-9, atol=1e-12 * np.abs(g).max())
        for j in range(3):
            i = rig.pk.material_names.index(f"fog{j}")
            assert ref[i, abi.GRAD_SIGMA_T] != 0.0, j
    finally:
        rig.close()
