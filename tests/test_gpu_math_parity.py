"""What the per-sample gate of the device-vs-oracle comparisons leaves unexplained.

The parity tests accept a small fraction of samples that differ beyond 1e-4: the device's
float transcendentals (CUDA's sinf, expf, powf, ...) and the host libm's differ in the last
ulp now and then, and a later comparison against a random number or a threshold can flip
on that ulp.  Here both sides take the SAME functions — the device's per-scene kernels
compiled with PTR_WIDE_MATH and the oracle's wide twin, both evaluating each float
transcendental in double and rounding once — and every sample agrees.  The residual of
the default comparison is measured beside it, so the two numbers bracket the cause.
"""
import numpy as np
import pytest

from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import CudaEngine

pytestmark = pytest.mark.gpu


def _cases():
    sc_m, st_m, _ = scenes.media_scene(spectral=False)
    sc_g, st_g, _ = scenes.mesh_scene(level=3, instances=4, env_size=(128, 64))
    return {
        "cornell-mis": (*scenes.cornell(direct="mis"), 64, 64, 8),
        "media-rgb": (sc_m, st_m, 48, 48, 8),
        "mesh-ggx-sky": (sc_g, st_g, 48, 27, 8),
    }


def _close(a, b):
    return (np.abs(a - b) <= 1e-4 * np.maximum(1.0, np.abs(b))).all(axis=-1)


@pytest.mark.parametrize("case", ["cornell-mis", "media-rgb", "mesh-ggx-sky"])
def test_same_transcendentals_give_the_same_samples(monkeypatch, oracle_lib, case):
    sc, st, W, H, spp = _cases()[case]
    r, pk = Compiler().compile(sc, st)
    rates = {}
    for wide in (False, True):
        if wide:
            monkeypatch.setenv("PTR_SPEC_DEFINES", "-DPTR_WIDE_MATH")
        else:
            monkeypatch.delenv("PTR_SPEC_DEFINES", raising=False)
        eng = CudaEngine(0)
        try:
            eng.register_scene(pk)
            eng.load_renderer(r)
            eng.specialize()
            eng.pin_reset_salt(11)
            dev = eng.render_samples(W, H, spp)
        finally:
            eng.close()
        o = oracle_lib.render(pk, r, W, H, spp, salt=11, keep_samples=True, variant="wide" if wide else "")
        rates["wide" if wide else "default"] = 1.0 - _close(dev, o["samples"]).mean()
    print(f"{case}: samples beyond 1e-4 - default math {rates['default']:.2e}, same math {rates['wide']:.2e}")
    assert rates["default"] <= 0.01
    assert rates["wide"] == 0.0, rates
