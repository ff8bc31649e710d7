"""The rough dielectric occupant (materials/rough_dielectric/rough_dielectric.glsl) in the
oracle, against the properties its reference test pins (rough_dielectric.test.ts):

* weight * pdf = eval * |cos| per sample on both lobes, and the sampler's pdf equals the
  pdf query (the agreement MIS needs), over both interface directions (entering glass,
  eta = 1/1.5; leaving it, eta = 1.5, where total internal reflection truncates the
  transmission lobe), three inclinations and three roughnesses;
* chi-square of the sampled directions' histogram over the whole sphere against the pdf
  integrated per cell (an edge at cos = 0, where the lobes meet);
* eta^2-aware reciprocity f(wi, wo; eta) = eta^2 f(-wo, -wi; 1/eta) for transmission and
  plain reciprocity for reflection;
* the index-matched interface is exactly the delta pass-through;
* eval covers the sampler's support: the mean weight equals the quadrature of eval |cos|;
* energy: the albedo with the transmitted part's eta^2 undone never exceeds 1 and falls
  with roughness.

The oracle's arithmetic is binary32, so the tolerances are float32's; the GPU parity tests
compare the device occupant with this one sample for sample.
"""
import math

import numpy as np
import pytest

ETAS = [("enter", 1.0, 1.5), ("exit", 1.5, 1.0)]     # (name, n_i, n_t): eta = n_i / n_t


def _dir(cos_t, phi):
    cos_t = np.asarray(cos_t, np.float64)
    s = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    return np.stack([s * np.cos(phi), s * np.sin(phi), cos_t], axis=-1)


def _alpha(r):
    return max(1e-3, r * r)


@pytest.mark.parametrize("interface", ETAS, ids=[e[0] for e in ETAS])
@pytest.mark.parametrize("cos_o", [0.9, 0.5, 0.1])
@pytest.mark.parametrize("roughness", [0.1, 0.4, 0.8])
def test_triple_and_pdf_agreement(oracle_lib, interface, cos_o, roughness):
    _, n_i, n_t = interface
    a = _alpha(roughness)
    wo = _dir(cos_o, 0.0)
    u = np.random.RandomState(17).rand(8192, 3)
    wi, w, pdf, flags = oracle_lib.rough_dielectric_sample(a, n_i, n_t, wo, u)
    live = pdf > 0
    assert live.sum() > 4000
    f, q = oracle_lib.rough_dielectric_eval(a, n_i, n_t, wi[live], wo)
    lhs = w[live, 0].astype(np.float64) * pdf[live]
    rhs = f[:, 0].astype(np.float64) * np.abs(wi[live, 2])
    ok = rhs > 1e-6 * rhs.max()
    # binary32: the half vector is recovered from (wi, wo) to ~1e-7, which D, peaked as
    # 1 / (sin^2 theta_h + alpha^2)^2, amplifies to ~7e-3 at alpha = 0.01 (r = 0.1)
    tol = 1e-2 if roughness < 0.2 else 1e-3
    assert np.max(np.abs(lhs[ok] - rhs[ok]) / rhs[ok]) < tol
    assert np.max(np.abs(q - pdf[live]) / pdf[live]) < tol
    if not (n_i > n_t and cos_o == 0.1):   # total internal reflection leaves no transmission
        assert (wi[live, 2] < 0).any()


def _chi2_crit(dof, z=3.0902):
    t = 1 - 2 / (9 * dof) + z * math.sqrt(2 / (9 * dof))
    return dof * t ** 3


@pytest.mark.parametrize("interface", ETAS, ids=[e[0] for e in ETAS])
@pytest.mark.parametrize("cos_o", [0.9, 0.5, 0.1])
@pytest.mark.parametrize("roughness", [0.4, 0.8])
def test_histogram_matches_pdf(oracle_lib, interface, cos_o, roughness):
    _, n_i, n_t = interface
    a = _alpha(roughness)
    wo = _dir(cos_o, 0.0)
    n = 1 << 17
    u = np.random.RandomState(987654 + int(cos_o * 1000) + int(roughness * 100)).rand(n, 3)
    wi, w, pdf, flags = oracle_lib.rough_dielectric_sample(a, n_i, n_t, wo, u)
    live = w[:, 0] > 0
    cb, pb = 16, 24
    row = np.minimum(cb - 1, np.floor((wi[live, 2] + 1) / 2 * cb)).astype(int)
    phi = np.arctan2(wi[live, 1], wi[live, 0])
    col = np.minimum(pb - 1, np.floor((phi + np.pi) / (2 * np.pi) * pb)).astype(int)
    counts = np.bincount(row * pb + col, minlength=cb * pb).astype(np.float64)
    # expected counts: midpoint quadrature of the pdf query, 48 x 48 probes per cell
    k = 48
    cgrid = -1 + (np.arange(cb * k) + 0.5) * (2.0 / (cb * k))
    pgrid = -np.pi + (np.arange(pb * k) + 0.5) * (2 * np.pi / (pb * k))
    cc, pp = np.meshgrid(cgrid, pgrid, indexing="ij")
    _, q = oracle_lib.rough_dielectric_eval(a, n_i, n_t, _dir(cc.ravel(), pp.ravel()), wo)
    cell = (2.0 / (cb * k)) * (2 * np.pi / (pb * k))
    mass = q.astype(np.float64).reshape(cb, k, pb, k).sum(axis=(1, 3)) * cell
    expected = n * mass.ravel()
    rejects, reject_e = n - live.sum(), n - expected.sum()
    big = expected >= 5
    chi2 = float((((counts - expected) ** 2)[big] / expected[big]).sum())
    cells = int(big.sum())
    pooled_e, pooled_o = expected[~big].sum(), counts[~big].sum()
    if reject_e >= 5:
        chi2 += (rejects - reject_e) ** 2 / reject_e
        cells += 1
    else:
        pooled_e += max(reject_e, 0.0)
        pooled_o += rejects
    if pooled_e >= 5:
        chi2 += (pooled_o - pooled_e) ** 2 / pooled_e
        cells += 1
    assert chi2 < _chi2_crit(cells - 1), (chi2, cells)


def test_reciprocity(oracle_lib):
    rng = np.random.RandomState(31337)
    n = 8000
    r = 0.05 + 0.9 * rng.rand()
    a = _alpha(r)
    wo = _dir(0.05 + 0.94 * rng.rand(n), 2 * np.pi * rng.rand(n))
    wi = _dir(-(0.05 + 0.94 * rng.rand(n)), 2 * np.pi * rng.rand(n))     # below: transmission
    f, _ = oracle_lib.rough_dielectric_eval(a, 1.0, 1.5, wi, wo)
    g, _ = oracle_lib.rough_dielectric_eval(a, 1.5, 1.0, -wo, -wi)
    eta2 = (1.0 / 1.5) ** 2
    ok = f[:, 0] > 0
    assert ok.sum() > 1000
    # binary32: relative to the value, plus an absolute floor for values near zero (the
    # reference's float64 check bounds the difference by 1e-9 max(1, f))
    diff = np.abs(f[ok, 0].astype(np.float64) - eta2 * g[ok, 0])
    assert (diff <= 1e-3 * f[ok, 0] + 1e-5 * f[ok, 0].max()).all()
    b = _dir(0.05 + 0.94 * rng.rand(n), 2 * np.pi * rng.rand(n))         # reflection: plain
    f2, _ = oracle_lib.rough_dielectric_eval(a, 1.0, 1.5, b, wo)
    g2, _ = oracle_lib.rough_dielectric_eval(a, 1.0, 1.5, wo, b)
    ok = f2[:, 0] > 0
    diff = np.abs(f2[ok, 0].astype(np.float64) - g2[ok, 0])
    assert (diff <= 1e-4 * f2[ok, 0] + 1e-6 * f2[ok, 0].max()).all()


def test_index_matched_interface_is_the_delta_pass_through(oracle_lib):
    rng = np.random.RandomState(2718)
    wo = _dir(0.02 + 0.97 * rng.rand(500), 2 * np.pi * rng.rand(500))
    tint = (0.8, 0.7, 0.6)
    for k in range(0, 500, 50):
        wi, w, pdf, flags = oracle_lib.rough_dielectric_sample(0.2, 1.3, 1.3, wo[k], rng.rand(4, 3), tint)
        np.testing.assert_array_equal(wi, np.repeat(-wo[k:k + 1].astype(np.float32), 4, 0))
        np.testing.assert_array_equal(w, np.repeat(np.asarray([tint], np.float32), 4, 0))
        assert not pdf.any() and (flags == 2 | 4).all()      # transmission | delta
        f, q = oracle_lib.rough_dielectric_eval(0.2, 1.3, 1.3, _dir(-1 + 2 * rng.rand(8), 2 * np.pi * rng.rand(8)), wo[k])
        assert not f.any() and not q.any()


@pytest.mark.parametrize("interface", ETAS, ids=[e[0] for e in ETAS])
def test_eval_covers_the_sampler_support(oracle_lib, interface):
    _, n_i, n_t = interface
    for cos_o in (0.9, 0.5, 0.2):
        for r in (0.3, 0.6):
            a = _alpha(r)
            wo = _dir(cos_o, 0.0)
            _, w, _, _ = oracle_lib.rough_dielectric_sample(a, n_i, n_t, wo, np.random.RandomState(4242).rand(1 << 16, 3))
            A = w[:, 0].astype(np.float64).mean()
            nc, npp = 500, 250
            c = -1 + (np.arange(nc) + 0.5) * (2.0 / nc)
            p = -np.pi + (np.arange(npp) + 0.5) * (2 * np.pi / npp)
            cc, pp = np.meshgrid(c, p, indexing="ij")
            f, _ = oracle_lib.rough_dielectric_eval(a, n_i, n_t, _dir(cc.ravel(), pp.ravel()), wo)
            B = float((f[:, 0].astype(np.float64) * np.abs(cc.ravel())).sum() * (2.0 / nc) * (2 * np.pi / npp))
            assert abs(A - B) / A < 0.01, (interface[0], cos_o, r, A, B)


@pytest.mark.parametrize("interface", ETAS, ids=[e[0] for e in ETAS])
def test_energy_albedo_bounded_and_falling_with_roughness(oracle_lib, interface):
    _, n_i, n_t = interface
    eta = n_i / n_t
    for cos_o in (0.95, 0.7, 0.4, 0.15):
        prev = np.inf
        for r in (0.05, 0.2, 0.5, 0.7):
            wi, w, _, _ = oracle_lib.rough_dielectric_sample(_alpha(r), n_i, n_t, _dir(cos_o, 0.0),
                                                             np.random.RandomState(777).rand(1 << 16, 3))
            up = wi[:, 2] > 0
            A = (w[up, 0].astype(np.float64).sum() + w[~up, 0].astype(np.float64).sum() / (eta * eta)) / len(w)
            assert A < 1.002 and A < prev * 1.002, (interface[0], cos_o, r, A, prev)
            prev = A
