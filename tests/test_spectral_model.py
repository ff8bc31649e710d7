"""The spectral colour model on the host (no GPU): lifts, blackbody, sampling densities."""
import numpy as np
import pytest

from pathtracerglsl_b200 import abi
from pathtracerglsl_b200.spectral import (LAMBDA_MAX, LAMBDA_MIN, MissingSpectralData, SpectralModel,
                                          wavelength_density, wavelength_sample)

LAM = np.linspace(LAMBDA_MIN, LAMBDA_MAX, 47001)


@pytest.fixture(scope="module")
def model():
    return SpectralModel.bundled()


@pytest.mark.parametrize("rgb", [(0.7, 0.5, 0.3), (0.75, 0.25, 0.25), (0.25, 0.75, 0.25), (0.9, 0.6, 0.3),
                                 (0.3, 0.6, 0.9)])
def test_reflectance_lift_round_trips_under_d65(model, rgb):
    """The Jakob-Hanika model's defining property: the lifted reflectance, lit by D65 and
    seen through the CIE sensor, returns the authored RGB."""
    rho = model.eval(model.reflectance(rgb), LAM)
    d65 = model.curves_at(LAM)[:, 3]
    out = np.trapezoid((rho * d65)[:, None] * model.sensor(LAM), LAM, axis=0)
    np.testing.assert_allclose(out, rgb, atol=1e-3)


def test_emission_and_coefficient_lifts(model):
    e = model.emission((1.0, 0.8, 0.6))
    out = np.trapezoid(model.eval(e, LAM)[:, None] * model.sensor(LAM), LAM, axis=0)
    np.testing.assert_allclose(out, (1.0, 0.8, 0.6), atol=1e-3)
    c = model.coefficient((0.5, 1.0, 2.0))
    assert c.kind == abi.SPEC_LIFTED and abs(c.scale - 4.0) < 1e-6
    grey = model.coefficient((2.0, 2.0, 2.0))
    assert grey.kind == abi.SPEC_GREY and grey.scale == 2.0
    assert model.reflectance((0.0, 0.0, 0.0)).kind == abi.SPEC_GREY


def test_blackbody_has_unit_reference_y(model):
    bb = model.blackbody(3000.0, 1.0)
    y = np.trapezoid(model.eval(bb, LAM) * model.curves_at(LAM)[:, 1], LAM) / model.cie_y_integral
    assert abs(y - 1.0) < 1e-4
    rgb = model.blackbody_rgb(3000.0)
    assert rgb[0] > rgb[1] > rgb[2] > 0       # warm: red > green > blue


@pytest.mark.parametrize("kind,lo,hi", [("visible", 360.0, 830.0), ("visible", 380.0, 780.0), ("uniform", 380.0, 780.0)])
def test_wavelength_densities_normalised_and_sampled(kind, lo, hi):
    lam = np.linspace(lo, hi, 40001)
    assert abs(np.trapezoid(wavelength_density(lam, kind, lo, hi), lam) - 1.0) < 1e-6
    for u in (0.0, 0.3, 0.999):
        ls, ps = wavelength_sample(u, kind, lo, hi)
        assert np.all((ls >= lo - 1e-6) & (ls <= hi + 1e-6))
        np.testing.assert_allclose(ps, wavelength_density(ls, kind, lo, hi), rtol=1e-9)


def test_sensor_constants(model):
    assert abs(model.cie_y_integral - 106.857) < 1e-2
    white = np.trapezoid(model.curves_at(LAM)[:, 3:4] * model.sensor(LAM), LAM, axis=0)
    np.testing.assert_allclose(white, 1.0, atol=5e-4)       # D65 is the sensor's white


def test_missing_node_fails_by_name(model):
    with pytest.raises(MissingSpectralData, match="coefficients.bin"):
        model.coefficients((0.11, 0.95, 0.42))
