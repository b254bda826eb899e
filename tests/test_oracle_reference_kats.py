"""The oracle's BSDFs pinned on the reference's own unit tests (read as
text; values and bounds as those tests state them):

  Tests/libgonzalesTests/FresnelTests.swift     dielectric Fresnel at normal
      incidence (glass 0.04, water), no boundary, grazing, total internal
      reflection, range, monotonicity, clamping of cos > 1;
  Tests/libgonzalesTests/BsdfTests.swift        diffuse value R / pi and
      upper-hemisphere samples; dielectric with eta 1 is black, smooth /
      rough specularity, specular sampling reflects for small u0 and
      transmits for large u0;
  Tests/libgonzalesTests/Coated.swift           a coated diffuse (eta 1,
      alpha 0.001, red base, thickness 0) evaluated at wo = (0, 0, 1),
      wi = (0, 0.1, 1) has red in (0.2, 0.4) and no green or blue;
  Tests/libgonzalesTests/TrowbridgeReitzTests.swift  alpha 0.0005 is smooth,
      0.5 is not; getAlpha(0.25) = 0.5 (the remapping the materials apply).

The Fresnel term is read through the smooth dielectric's sample: its
reflection probability is F(cos theta).

The sampling, interaction and filter helpers the integrator uses are pinned
the same way:

  Tests/libgonzalesTests/SamplingTests.swift    power heuristic values,
      concentric disk centre and unit circle, cosine hemisphere length and
      upper half;
  Tests/libgonzalesTests/InteractionTests.swift offset origin on the
      direction's side of the normal; shadow spawn toward the target with
      tHit in (0.99, 1);
  Tests/libgonzalesTests/FilterTests.swift      Gaussian filter (support 2,
      sigma 1): centre above edge, non-negative, symmetric, samples inside
      the support with positive density."""
import math

import numpy as np
import pytest

from oracle import pyoracle as O


def fresnel(cos_theta, eta):
    """F through the specular dielectric: reflection chosen with probability F."""
    p = O.bsdf_params(3, eta=eta, roughness=0.0)
    s = math.sqrt(max(0.0, 1.0 - cos_theta * cos_theta))
    wo = [s, 0.0, cos_theta]
    ok, f, wi, pdf = O.bsdf_sample(p, wo, [0.0, 0.5, 0.5])
    if eta == 1.0:
        # no boundary: always transmitted (reflection probability 0)
        return 0.0 if (ok and wi[2] * cos_theta < 0) else 1.0
    assert ok and wi[2] * cos_theta > 0  # u0 = 0 < F picks the reflection
    return pdf


def test_fresnel_normal_incidence():
    assert abs(fresnel(1.0, 1.5) - 0.04) <= 1e-4
    assert abs(fresnel(1.0, 1.33) - ((1 - 1.33) / (1 + 1.33)) ** 2) <= 1e-4


def test_fresnel_no_boundary():
    assert fresnel(1.0, 1.0) == 0.0
    assert fresnel(0.707, 1.0) == 0.0


def test_fresnel_grazing_and_total_internal_reflection():
    assert fresnel(0.001, 1.5) > 0.95
    assert abs(fresnel(-0.3, 1.5) - 1.0) <= 1e-6


def test_fresnel_range_and_monotonicity():
    for c in (-1.0, -0.5, -0.1, 0.1, 0.5, 0.7, 0.9, 1.0):
        for eta in (1.33, 1.5, 2.0, 2.5):
            r = fresnel(c, eta)
            assert -1e-6 <= r <= 1.0 + 1e-6
    prev = 0.0
    for i in range(10, 0, -1):
        r = fresnel(i / 10.0, 1.5)
        assert r >= prev - 1e-6
        prev = r


def test_diffuse_value_and_samples():
    p = O.bsdf_params(1, reflectance=(0.8, 0.4, 0.2))
    wi = np.array([0.5, 0.0, 1.0])
    wi /= np.linalg.norm(wi)
    f, _ = O.bsdf_eval(p, [0, 0, 1], wi)
    np.testing.assert_allclose(f, np.array([0.8, 0.4, 0.2]) / math.pi, atol=1e-5)
    for u in ((0.1, 0.2, 0.3), (0.5, 0.5, 0.5), (0.9, 0.1, 0.8)):
        ok, f, wi, pdf = O.bsdf_sample(O.bsdf_params(1, reflectance=(1, 1, 1)), [0, 0, 1], u)
        assert wi[2] >= 0 and pdf > 0


def test_dielectric_cases():
    wi = np.array([0.3, 0.0, 1.0])
    wi /= np.linalg.norm(wi)
    f, _ = O.bsdf_eval(O.bsdf_params(3, eta=1.0, roughness=0.25), [0, 0, 1], wi)
    assert np.all(f == 0)  # eta 1: no boundary, black
    smooth = O.bsdf_params(3, eta=1.5, roughness=0.0005 ** 2)  # alpha 0.0005
    rough = O.bsdf_params(3, eta=1.5, roughness=0.25)          # alpha 0.5
    assert O.bsdf_is_specular(smooth) and not O.bsdf_is_specular(rough)
    ok, f, wi, pdf = O.bsdf_sample(smooth, [0, 0, 1], [0.1, 0.5, 0.5])
    assert pdf > 0
    assert O.bsdf_sample(smooth, [0, 0, 1], [0.01, 0.5, 0.5])[2][2] > 0   # reflects
    assert O.bsdf_sample(smooth, [0, 0, 1], [0.99, 0.5, 0.5])[2][2] < 0   # transmits


def test_coated_diffuse_reference_case():
    # alpha 0.001 = sqrt(roughness) with roughness 1e-6; the coating's eta 1;
    # red base; thickness 0 (raised to the least normal float)
    p = O.bsdf_params(4, reflectance=(1.0, 0.0, 0.0), eta=1.0, roughness=1e-6, thickness=0.0)
    f, _ = O.bsdf_eval(p, [0.0, 0.0, 1.0], [0.0, 0.1, 1.0])
    assert 0.2 < f[0] < 0.4
    assert abs(f[1]) <= 1e-6 and abs(f[2]) <= 1e-6


def test_roughness_remapping():
    # getAlpha(0.25) = 0.5: a dielectric of roughness 0.25 has alpha 0.5, not smooth
    assert not O.bsdf_is_specular(O.bsdf_params(3, eta=1.5, roughness=0.25))
    # roughness 0.0005^2 gives alpha 0.0005 < 0.001: smooth
    assert O.bsdf_is_specular(O.bsdf_params(3, eta=1.5, roughness=0.0005 ** 2))


# --- Tests/libgonzalesTests/SamplingTests.swift -----------------------------


@pytest.mark.parametrize("f,g,want", [(1.0, 1.0, 0.5), (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 0.0),
                                      (2.0, 3.0, 4.0 / 13.0)])
def test_power_heuristic_known_values(f, g, want):
    assert abs(O.power_heuristic(f, g) - want) <= 1e-6


def test_power_heuristic_dominating_and_dominated():
    assert O.power_heuristic(100.0, 1.0) > 0.99
    assert O.power_heuristic(1.0, 100.0) < 0.01


def test_concentric_disk_center_and_unit_circle():
    c = O.concentric_disk(0.5, 0.5)
    assert abs(c[0]) <= 1e-6 and abs(c[1]) <= 1e-6
    for u in [(0.0, 0.0), (1.0, 0.0), (0.0, 1.0), (1.0, 1.0), (0.25, 0.75), (0.8, 0.2)]:
        d = O.concentric_disk(*u)
        assert d[0] * d[0] + d[1] * d[1] <= 1.0 + 1e-6, u


def test_cosine_hemisphere_unit_length_and_upper():
    v = O.cosine_hemisphere(0.3, 0.7)
    assert abs(np.linalg.norm(v.astype(np.float64)) - 1.0) <= 1e-5
    for u in [(0.1, 0.1), (0.5, 0.5), (0.9, 0.9), (0.0, 0.0)]:
        assert O.cosine_hemisphere(*u)[2] >= 0, u


# --- Tests/libgonzalesTests/InteractionTests.swift --------------------------


def test_offset_origin_follows_direction_side():
    p, n = [0, 0, 0], [0, 0, 1]
    assert O.offset_origin(p, n, [0, 0, 1])[2] > 0
    assert O.offset_origin(p, n, [0, 0, -1])[2] < 0


def test_spawn_to_target():
    o, d, t = O.spawn_to([0, 0, 0], [10, 0, 0])
    assert d[0] > 0
    assert 0.99 < t < 1.0
    # the ray ends on the target at t = 1
    np.testing.assert_allclose(o + d, [10, 0, 0], atol=1e-5)


# --- Tests/libgonzalesTests/FilterTests.swift (GaussianFilter) ------------


def test_gaussian_filter_shape():
    ev = lambda x, y: O.gaussian_filter_evaluate(x, y, 1.0)
    assert ev(0, 0) > ev(1.5, 1.5)
    for x, y in [(0, 0), (1, 0), (0, 1), (1.9, 1.9)]:
        assert ev(x, y) >= 0
    assert abs(ev(0.5, 0.7) - ev(-0.5, -0.7)) <= 1e-6


def test_gaussian_filter_sample_within_support():
    for u in [(0.1, 0.1), (0.5, 0.5), (0.9, 0.9)]:
        (x, y), dens = O.gaussian_filter_sample(u[0], u[1], 2.0, 1.0)
        assert abs(x) <= 2.0 + 1e-6 and abs(y) <= 2.0 + 1e-6
        assert dens > 0
