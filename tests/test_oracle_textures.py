"""CPU checks of the oracle's textured renderer (the checker of the GPU
adjoint): constant textures equal to a material's albedo reproduce the plain
render bit for bit, scaling emission by 2 doubles every film sum exactly
(every emission enters a path's radiance linearly; x2 is exact in FP32), and
changing one texel channel changes only that channel of the pixels it
reaches."""
import numpy as np

from gonzales_b200 import adjoint as A
from oracle import pyoracle as O


def _scene():
    sb, mats = A.adjoint_box_scene()
    return sb.build(), mats


def _tex(mt, maps, texels, scale=1.0):
    return dict(material_texture=mt, maps=maps, texels=texels, emission_scale=scale)


def test_constant_textures_reproduce_plain_render():
    hs, mats = _scene()
    mt, maps = A.texture_maps(mats, len(hs.materials))
    R = 8
    tex = np.zeros((2, R, R, 3), np.float32)
    for t, m in enumerate(mats):
        tex[t] = np.asarray(hs.materials[m]["albedo"], np.float32)
    p = O.render_params(24, 20, 4, max_depth=4, rr_min_bounce=2)
    plain = O.render(hs, p, threads=4)
    textured = O.render(hs, p, threads=4, textures=_tex(mt, maps, tex))
    for a, b in zip(plain[:3], textured[:3]):
        assert a.tobytes() == b.tobytes()


def test_emission_scale_is_linear():
    hs, mats = _scene()
    mt, maps = A.texture_maps(mats, len(hs.materials))
    tex = A.ground_truth_textures(res=16)
    p = O.render_params(24, 20, 4, max_depth=4, rr_min_bounce=4)
    one = O.render(hs, p, threads=4, textures=_tex(mt, maps, tex, 1.0))
    two = O.render(hs, p, threads=4, textures=_tex(mt, maps, tex, 2.0))
    assert (2 * one[0]).tobytes() == two[0].tobytes()
    assert one[2].tobytes() == two[2].tobytes()


def test_texel_value_changes_only_reached_pixels():
    hs, mats = _scene()
    mt, maps = A.texture_maps(mats, len(hs.materials))
    tex = A.ground_truth_textures(res=4)
    p = O.render_params(32, 32, 2, max_depth=1, rr_min_bounce=1)
    base = O.render(hs, p, threads=4, textures=_tex(mt, maps, tex))
    bumped = tex.copy()
    bumped[0, 3, 3, 0] += 0.25  # front-right floor texel (x, z) in [0.75, 1)^2, red channel
    moved = O.render(hs, p, threads=4, textures=_tex(mt, maps, bumped))
    diff = moved[0] != base[0]
    assert diff[..., 0].any() and not diff[..., 1].any() and not diff[..., 2].any()
