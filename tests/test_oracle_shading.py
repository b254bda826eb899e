"""The oracle's surface interaction with vertex normals and UVs
(Triangle.computeSurfaceInteraction, Shape/Triangle.swift:386-452): the
shading normal interpolated from the vertex normals, dpdu from the UVs.

  - vertex normals equal to the face normals (unshared vertices) shade like
    no normals at all (the same image up to rounding);
  - smooth normals on a sphere change the image (the shading frame and the
    light-sample cosine follow the interpolated normal) but not its overall
    brightness by much;
  - the renders are deterministic."""
import numpy as np

from gonzales_b200 import scenes
from gonzales_b200.scene import SceneBuilder
from oracle import pyoracle as O


def _facet_scene(with_normals):
    rng = np.random.default_rng(4)
    sb = SceneBuilder()
    scenes._room(sb, rng)
    sp, st = scenes.icosphere(1)
    pts = (sp * 0.2 + np.array([0.5, 0.2, 0.5]))[st.reshape(-1)]
    tris = np.arange(len(pts)).reshape(-1, 3)
    # the interaction's geometric normal is cross(p0 - p2, p1 - p2)
    fn = np.cross(pts[tris[:, 0]] - pts[tris[:, 2]], pts[tris[:, 1]] - pts[tris[:, 2]])
    fn /= np.linalg.norm(fn, axis=1, keepdims=True)
    nrm = np.repeat(fn, 3, axis=0) if with_normals else None
    sb.add_mesh(pts, tris, sb.add_material((0.6, 0.5, 0.4)), normals=nrm)
    lp, lt = scenes._quad((0.35, 0.999, 0.35), (0.65, 0.999, 0.35), (0.65, 0.999, 0.65), (0.35, 0.999, 0.65))
    sb.add_area_light(lp, lt, (15.0, 11.0, 4.0))
    return sb.build()


def test_face_normals_shade_like_no_normals():
    p = O.render_params(48, 48, 8, max_depth=4, rr_min_bounce=3)
    a = O.render(_facet_scene(False), p)
    b = O.render(_facet_scene(True), p)
    np.testing.assert_allclose(b[0].sum() / b[2].sum(), a[0].sum() / a[2].sum(), rtol=1e-2)
    assert np.isclose(a[0], b[0], rtol=1e-3, atol=1e-4).mean() > 0.9


def test_smooth_normals_change_the_image_deterministically():
    sb = scenes.smooth_box_scene()
    hs = sb.build()
    p = O.render_params(48, 48, 8, max_depth=4, rr_min_bounce=3)
    a = O.render(hs, p)
    b = O.render(hs, p)
    assert np.array_equal(a[0], b[0])
    for m in hs.meshes:
        m.normals = None
        m.uvs = None
    c = O.render(hs, p)
    assert not np.allclose(a[0], c[0])
    np.testing.assert_allclose(a[0].sum() / a[2].sum(), c[0].sum() / c[2].sum(), rtol=0.1)
    assert np.isfinite(a[0]).all()
