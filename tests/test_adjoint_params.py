"""The adjoint's parameter space on the host (no GPU): read, write and live slots."""
import numpy as np

from pathtracerglsl_b200 import abi, adjoint, scenes
from pathtracerglsl_b200.compiler import Compiler


def test_param_table_roundtrip_and_mask():
    sc, st, _ = scenes.adjoint_scene(0)
    r, pk = Compiler().compile(sc, st)
    mask = adjoint.live_mask(pk)
    theta = adjoint.param_table(pk)
    names = pk.material_names
    fog = names.index("fog")
    assert mask[fog, abi.GRAD_SIGMA_T] and mask[fog, abi.GRAD_MEDIUM_ALBEDO] and mask[fog, abi.GRAD_HG_G]
    assert abs(theta[fog, abi.GRAD_SIGMA_T] - 2.0) < 1e-6 and abs(theta[fog, abi.GRAD_MEDIUM_ALBEDO] - 0.9) < 1e-6
    # 64 spheres + 3 walls + the medium, each with its model's full set: Lambert albedo (3),
    # GGX F0 (3) + alpha, dielectric transmittance (3) + IOR, the medium's sigma_t, albedo
    # and g (about 260); the light's synthesized material is not a parameter
    counts = {"lambert": 3, "ggx": 4, "dielectric": 4, "none": 3}
    assert mask.sum() == sum(counts[m["model"]] for m in sc["materials"].values())
    assert 240 <= mask.sum() <= 270
    t2 = theta.copy()
    t2[mask] *= 1.1
    pk2 = adjoint.with_params(pk, t2)
    back = adjoint.param_table(pk2)
    np.testing.assert_allclose(back[mask], t2[mask], rtol=1e-6)
    # untouched: the original tables, the shapes of the copy
    np.testing.assert_allclose(adjoint.param_table(pk)[mask], theta[mask])
    assert pk2.regions.shape == pk.regions.shape


def test_l2_loss_derivative():
    a = np.random.RandomState(0).rand(4, 5, 3).astype(np.float32)
    b = np.zeros_like(a)
    loss, d = adjoint.l2_loss(a, b)
    assert abs(loss - float((a.astype(np.float64) ** 2).mean())) < 1e-12
    np.testing.assert_allclose(d, 2 * a / a.size, rtol=1e-6)
