"""Differentiable rendering: path-replay adjoint of the wavefront integrator.

The scene is the box scene with albedo textures on the floor and the back
wall and a scalar scale on the light's emission.  A render is a function of
the texels and the scale; `DifferentiableRenderer.forward` returns the image
(film sums / film weights) and `backward` maps dLoss/dImage to dLoss/dtexel
and dLoss/dscale with gzg_renderer_adjoint (one primal pass + one replay per
wave, no stored path graph).  `render` wraps the pair as a
torch.autograd.Function.

Russian roulette is not differentiated (its survival probability depends on
the throughput), so adjoint renders trace every path to max_depth:
rr_min_bounce = max_depth.
"""
import ctypes as C
import math

import numpy as np

from . import _ffi as F
from .accel import Renderer, _stream_handle
from .scene import SceneBuilder
from .scenes import _box, _quad, value_noise

TEXTURE_RES = 256
# planar maps (origin, u axis, v axis) of the two textures
FLOOR = ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0))
BACK_WALL = ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0))


def adjoint_box_scene(seed=0xB0):
    """The box scene with the floor and the back wall as their own materials
    (1 and 2); material 0 (ceiling and side walls) is what area-light hits
    scatter with.  Returns (builder, [floor material, back-wall material])."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    base = rng.uniform(0.1, 0.8, 3)
    others = [
        _quad((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)),   # ceiling y=1
        _quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)),   # left x=0
        _quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)),   # right x=1
    ]
    m_walls = sb.add_material(base)
    m_floor = sb.add_material(base)
    m_back = sb.add_material(base)
    pts = np.concatenate([w[0] for w in others])
    tris = np.concatenate([w[1] + 4 * i for i, w in enumerate(others)])
    sb.add_mesh(pts, tris, m_walls)
    fp, ft = _quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1))
    sb.add_mesh(fp, ft, m_floor)
    bp, bt = _quad((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0))
    sb.add_mesh(bp, bt, m_back)
    for cx, cz in ((0.3, 0.35), (0.68, 0.62)):
        size = rng.uniform(0.2, 0.35)
        ang = rng.uniform(0, math.pi / 2)
        p, t = _box(size, ang, (cx, size / 2.0 + 1e-4, cz))
        sb.add_mesh(p, t, sb.add_material(rng.uniform(0.1, 0.8, 3)))
    lp, lt = _quad((0.35, 0.999, 0.35), (0.65, 0.999, 0.35), (0.65, 0.999, 0.65), (0.35, 0.999, 0.65))
    sb.add_area_light(lp, lt, (15.0, 11.0, 4.0))
    return sb, [m_floor, m_back]


def texture_bindings(materials):
    """gzg_texture_binding records: floor texture 0, back-wall texture 1."""
    out = (F.TextureBinding * len(materials))()
    for k, (m, (o, u, v)) in enumerate(zip(materials, (FLOOR, BACK_WALL))):
        out[k] = F.TextureBinding(m, 0, (C.c_float * 3)(*o), (C.c_float * 3)(*u), (C.c_float * 3)(*v))
    return out


def texture_maps(materials, n_materials):
    """The same bindings for the oracle: per-material texture index and maps."""
    mt = np.full(n_materials, -1, np.int32)
    maps = np.zeros((len(materials), 9), np.float32)
    for k, (m, (o, u, v)) in enumerate(zip(materials, (FLOOR, BACK_WALL))):
        mt[m] = k
        maps[k] = np.concatenate([o, u, v])
    return mt, maps


def ground_truth_textures(seed=0xC4, res=TEXTURE_RES):
    """Seeded albedo textures in [0.1, 0.8]: 3-octave value noise per channel
    plus a checker of period res / 8 texels."""
    iy, ix = np.meshgrid(np.arange(res), np.arange(res), indexing="ij")
    period = max(1, res // 8)
    out = np.zeros((2, res, res, 3), np.float32)
    for t in range(2):
        for c in range(3):
            p = np.stack([ix / res * 2.0, iy / res * 2.0, np.full(ix.shape, 0.37 * (3 * t + c))], -1).reshape(-1, 3)
            n = value_noise(p, seed + 7 * t + c).reshape(res, res)
            checker = ((ix // period + iy // period) % 2) * 0.15
            out[t, :, :, c] = np.clip(0.4 + 0.25 * n + checker - 0.075, 0.1, 0.8)
    return out


class DifferentiableRenderer:
    """Forward renders and adjoint passes of one scene with bound textures.

    texels: torch CUDA float32 tensor (T, R, R, 3), read at every render
    (update it in place between renders); emission scale: a Python float.
    forward_only=True allows roulette (no adjoint is then exact)."""

    def __init__(self, accel, params, materials, resolution=TEXTURE_RES, forward_only=False):
        if not forward_only and params.rr_min_bounce < params.max_depth:
            raise ValueError("adjoint renders need rr_min_bounce >= max_depth (roulette is not differentiated)")
        self.params = params
        self.materials = list(materials)
        self.resolution = resolution
        self.bindings = texture_bindings(self.materials)
        self.renderer = Renderer(accel, params)
        self._bound = None

    def bind(self, texels, emission_scale):
        key = (texels.data_ptr(), float(emission_scale))
        if key != self._bound:
            if tuple(texels.shape) != (len(self.materials), self.resolution, self.resolution, 3) or \
                    not texels.is_contiguous() or texels.dtype.itemsize != 4 or not texels.is_floating_point():
                raise ValueError("texels must be a contiguous float32 (%d, %d, %d, 3) tensor"
                                 % (len(self.materials), self.resolution, self.resolution))
            F.check(F.lib().gzg_renderer_set_textures(self.renderer.handle, self.bindings, len(self.materials),
                                                      self.resolution, texels.data_ptr(), float(emission_scale)))
            self._bound = key

    def films(self, texels, emission_scale, f64=False, stream=None):
        """Film sums (rgb (H, W, 3), w (H, W)) of one render."""
        import torch

        self.bind(texels, emission_scale)
        H, W = self.params.film_height, self.params.film_width
        dt = torch.float64 if f64 else torch.float32
        rgb = torch.zeros((H, W, 3), dtype=dt, device=texels.device)
        w = torch.zeros((H, W), dtype=dt, device=texels.device)
        if f64:
            F.check(F.lib().gzg_renderer_render_f64(self.renderer.handle, rgb.data_ptr(), None, w.data_ptr(),
                                                    _stream_handle(stream)))
        else:
            self.renderer.render(rgb, w, stream=stream)
        return rgb, w

    def forward(self, texels, emission_scale, f64=False, stream=None):
        """(image (H, W, 3), film weights (H, W))."""
        rgb, w = self.films(texels, emission_scale, f64=f64, stream=stream)
        return rgb / w[..., None], w

    def backward(self, grad_image, film_w, texels, emission_scale, stream=None):
        """dLoss/dtexels (like texels) and dLoss/demission_scale (float64
        0-d tensor) for dLoss/dImage = grad_image (H, W, 3)."""
        import torch

        self.bind(texels, emission_scale)
        g = grad_image.detach().to(torch.float32).contiguous()
        fw = film_w.detach().to(torch.float32).contiguous()
        d_tex = torch.zeros_like(texels)
        d_em = torch.zeros((), dtype=torch.float64, device=texels.device)
        F.check(F.lib().gzg_renderer_adjoint(self.renderer.handle, g.data_ptr(), fw.data_ptr(), d_tex.data_ptr(),
                                             d_em.data_ptr(), _stream_handle(stream)))
        return d_tex, d_em

    def close(self):
        self.renderer.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _function():
    import torch

    class RenderFunction(torch.autograd.Function):
        """image = render(texels, emission_scale); backward by path replay."""

        @staticmethod
        def forward(ctx, texels, emission_scale, dr):
            scale = float(emission_scale.detach().item())
            image, w = dr.forward(texels.detach(), scale)
            ctx.dr = dr
            ctx.scale = scale
            ctx.scale_dtype = emission_scale.dtype
            ctx.save_for_backward(texels, w)
            return image

        @staticmethod
        def backward(ctx, grad_image):
            texels, w = ctx.saved_tensors
            d_tex, d_em = ctx.dr.backward(grad_image, w, texels.detach(), ctx.scale)
            return d_tex, d_em.to(ctx.scale_dtype), None

    return RenderFunction


_RENDER_FUNCTION = None


def render(texels, emission_scale, dr):
    """Differentiable render: torch.autograd sees texels (T, R, R, 3) and the
    0-d emission_scale tensor."""
    global _RENDER_FUNCTION
    if _RENDER_FUNCTION is None:
        _RENDER_FUNCTION = _function()
    return _RENDER_FUNCTION.apply(texels, emission_scale, dr)
