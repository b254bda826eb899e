"""The oracle's dielectric, coated-diffuse, conductor and coated-conductor BSDFs
(Bsdf/DielectricBsdf.swift, Bsdf/LayeredBsdf.swift with
Bsdf/CoatedDiffuseBsdf.swift and Bsdf/CoatedConductorBsdf.swift,
Bsdf/MicrofacetReflection.swift with Reflection/FresnelConductor.swift) checked through
properties the reference's forms imply; the reference ships no golden
vectors for them:

  - a smooth dielectric splits by the Fresnel term (0.04 at normal incidence
    for eta 1.5) and scales transmitted radiance by 1 / eta^2;
  - a rough dielectric's sample returns the value and density its evaluate
    and probabilityDensity give for the sampled direction (from outside; from
    inside the reference's half-vector sampling flips the half vector into
    the outgoing hemisphere, TrowbridgeReitzDistribution.swift:28-38, which
    its evaluation does not, so the two differ there by design);
  - the density integrates to the fraction of valid samples;
  - a coated diffuse over a black base is its coating alone, reflects like
    the coating when the coating sample reflects, has a density no lower than
    the uniform floor 0.1 / (4 pi), and reflects no more than it receives;
  - a conductor reflects the conductor Fresnel term at normal incidence, its
    sample agrees with its evaluation and its density integrates to the valid
    fraction; a coated conductor behaves like the coated diffuse above.
"""
import math

import numpy as np
import pytest

from oracle import pyoracle as O


def _upper(rng, n):
    d = rng.normal(size=(n, 3))
    d[:, 2] = np.abs(d[:, 2])
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def test_smooth_dielectric_fresnel_split():
    p = O.bsdf_params(3, eta=1.5, roughness=0.0)
    assert O.bsdf_is_specular(p)
    ok, f, wi, pdf = O.bsdf_sample(p, [0, 0, 1], [0.01, 0.5, 0.5])
    assert ok and wi[2] == 1.0
    np.testing.assert_allclose([f[0] * abs(wi[2]), pdf], [0.04, 0.04], rtol=1e-5)
    ok, f, wi, pdf = O.bsdf_sample(p, [0, 0, 1], [0.5, 0.5, 0.5])
    assert ok and wi[2] == -1.0
    np.testing.assert_allclose([f[0] * abs(wi[2]), pdf], [0.96 / 1.5 ** 2, 0.96], rtol=1e-5)
    # delta lobes: no value or density for given directions
    f, pdf = O.bsdf_eval(p, [0, 0, 1], [0, 0, 1])
    assert f[0] == 0.0 and pdf == 0.0


@pytest.mark.parametrize("rough", [0.05, 0.2, 0.5])
def test_rough_dielectric_sample_matches_evaluation(rough):
    p = O.bsdf_params(3, eta=1.5, roughness=rough)
    assert not O.bsdf_is_specular(p)
    rng = np.random.default_rng(7)
    n = 0
    for wo, u in zip(_upper(rng, 600), rng.random((600, 3))):
        ok, f, wi, pdf = O.bsdf_sample(p, wo, u)
        if not ok:
            continue
        fe, pe = O.bsdf_eval(p, wo, wi)
        np.testing.assert_allclose(fe, f, rtol=1e-4, atol=1e-7)
        assert abs(pe - pdf) <= 1e-4 * pdf + 1e-7
        n += 1
    assert n > 500


def test_rough_dielectric_density_integrates_to_valid_fraction():
    p = O.bsdf_params(3, eta=1.5, roughness=0.3)
    rng = np.random.default_rng(11)
    wo = np.array([0.3, 0.1, 0.8])
    wo /= np.linalg.norm(wo)
    n = 30000
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    vals = np.array([O.bsdf_eval(p, wo, x)[1] for x in d])
    integral = vals.mean() * 4 * math.pi
    se = vals.std() * 4 * math.pi / math.sqrt(n)
    valid = np.mean([O.bsdf_sample(p, wo, u)[0] for u in rng.random((n, 3))])
    assert abs(integral - valid) < 4 * se + 0.01, (integral, se, valid)


def test_coated_over_black_base_is_the_coating():
    coat = O.bsdf_params(3, eta=1.5, roughness=0.3)
    coated = O.bsdf_params(4, reflectance=(0, 0, 0), eta=1.5, roughness=0.3, thickness=0.01)
    rng = np.random.default_rng(3)
    for wo, wi in zip(_upper(rng, 200), _upper(rng, 200)):
        fc, _ = O.bsdf_eval(coated, wo, wi)
        fd, _ = O.bsdf_eval(coat, wo, wi)
        np.testing.assert_allclose(fc, fd, rtol=1e-6, atol=0)


def test_coated_reflects_like_its_coating_when_the_coating_reflects():
    coat = O.bsdf_params(3, eta=1.5, roughness=0.3)
    coated = O.bsdf_params(4, reflectance=(0.7, 0.5, 0.3), eta=1.5, roughness=0.3, thickness=0.01)
    rng = np.random.default_rng(5)
    seen = 0
    for wo, u in zip(_upper(rng, 400), rng.random((400, 3))):
        ok_d, fd, wid, pd = O.bsdf_sample(coat, wo, u)
        if not ok_d or wid[2] <= 0:
            continue
        ok_c, fc, wic, pc = O.bsdf_sample(coated, wo, u)
        assert ok_c
        np.testing.assert_array_equal(wic, wid)
        np.testing.assert_array_equal(fc, fd)
        assert pc == pd
        seen += 1
    assert seen > 5


def test_coated_is_deterministic_and_density_has_its_floor():
    p = O.bsdf_params(4, reflectance=(0.6, 0.5, 0.4), eta=1.5, roughness=0.2, thickness=0.01)
    rng = np.random.default_rng(9)
    floor = 0.1 / (4 * math.pi)
    for wo, wi in zip(_upper(rng, 100), rng.normal(size=(100, 3))):
        wi = wi / np.linalg.norm(wi)
        f1, p1 = O.bsdf_eval(p, wo, wi)
        f2, p2 = O.bsdf_eval(p, wo, wi)
        np.testing.assert_array_equal(f1, f2)
        assert p1 == p2
        assert p1 >= floor * (1 - 1e-6)
        assert np.all(f1 >= 0)


@pytest.mark.parametrize("rough", [0.05, 0.4])
def test_coated_reflects_at_most_what_it_receives(rough):
    p = O.bsdf_params(4, reflectance=(1, 1, 1), eta=1.5, roughness=rough, thickness=0.01)
    rng = np.random.default_rng(13)
    wo = np.array([0.2, -0.3, 0.9])
    wo /= np.linalg.norm(wo)
    acc = np.zeros(3)
    n = 8000
    for u in rng.random((n, 3)):
        ok, f, wi, pdf = O.bsdf_sample(p, wo, u)
        if ok and pdf > 0:
            acc += f * abs(wi[2]) / pdf
    albedo = acc / n
    assert np.all(albedo <= 1.02) and np.all(albedo > 0.2), albedo


def test_conductor_fresnel_at_normal_incidence():
    # alpha 1: D(z) = 1 / pi and G(z, z) = 1, so f(z, z) = F(0) / (4 pi) with
    # F(0) = ((n - 1)^2 + k^2) / ((n + 1)^2 + k^2) per channel
    eta, k = (0.2, 0.92, 1.1), (3.9, 2.45, 2.14)
    p = O.bsdf_params(5, conductor_eta=eta, conductor_k=k, conductor_roughness=1.0)
    f, pdf = O.bsdf_eval(p, [0, 0, 1], [0, 0, 1])
    n, kk = np.array(eta), np.array(k)
    f0 = ((n - 1) ** 2 + kk ** 2) / ((n + 1) ** 2 + kk ** 2)
    np.testing.assert_allclose(f * 4 * math.pi, f0, rtol=1e-5)
    assert not O.bsdf_is_specular(p)


@pytest.mark.parametrize("rough", [0.05, 0.3])
def test_conductor_sample_matches_evaluation(rough):
    p = O.bsdf_params(5, conductor_roughness=rough)
    rng = np.random.default_rng(17)
    n = 0
    for wo, u in zip(_upper(rng, 600), rng.random((600, 3))):
        ok, f, wi, pdf = O.bsdf_sample(p, wo, u)
        if not ok:
            continue
        fe, pe = O.bsdf_eval(p, wo, wi)
        np.testing.assert_allclose(fe, f, rtol=1e-5, atol=0)
        assert pe == pdf
        assert wi[2] > 0
        n += 1
    assert n > 450


def test_conductor_density_integrates_to_valid_fraction():
    p = O.bsdf_params(5, conductor_roughness=0.3)
    rng = np.random.default_rng(19)
    wo = np.array([0.5, -0.2, 0.7])
    wo /= np.linalg.norm(wo)
    n = 30000
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    vals = np.array([O.bsdf_eval(p, wo, x)[1] for x in d])
    integral = vals.mean() * 4 * math.pi
    se = vals.std() * 4 * math.pi / math.sqrt(n)
    valid = np.mean([O.bsdf_sample(p, wo, u)[0] for u in rng.random((n, 3))])
    assert abs(integral - valid) < 4 * se + 0.01, (integral, se, valid)


def test_coated_conductor_reflects_like_its_coating_when_the_coating_reflects():
    coat = O.bsdf_params(3, eta=1.5, roughness=0.2)
    cc = O.bsdf_params(6, reflectance=(0.9, 0.8, 0.5), eta=1.5, roughness=0.2, thickness=0.02,
                       conductor_roughness=0.3)
    rng = np.random.default_rng(23)
    seen = 0
    for wo, u in zip(_upper(rng, 400), rng.random((400, 3))):
        ok_d, fd, wid, pd = O.bsdf_sample(coat, wo, u)
        if not ok_d or wid[2] <= 0:
            continue
        ok_c, fc, wic, pc = O.bsdf_sample(cc, wo, u)
        assert ok_c
        np.testing.assert_array_equal(wic, wid)
        np.testing.assert_array_equal(fc, fd)
        seen += 1
    assert seen > 5


def test_coated_conductor_over_black_base_is_the_coating():
    coat = O.bsdf_params(3, eta=1.5, roughness=0.3)
    cc = O.bsdf_params(6, reflectance=(0, 0, 0), eta=1.5, roughness=0.3, thickness=0.01, conductor_roughness=0.2)
    rng = np.random.default_rng(29)
    for wo, wi in zip(_upper(rng, 200), _upper(rng, 200)):
        fc, pc = O.bsdf_eval(cc, wo, wi)
        fd, _ = O.bsdf_eval(coat, wo, wi)
        np.testing.assert_allclose(fc, fd, rtol=1e-6, atol=0)
        assert pc >= 0.1 / (4 * math.pi) * (1 - 1e-6)
