"""Pins the oracle (the CPU restatement used as checker) against the
reference's own known-answer tests and against published values.

  Tests/libgonzalesTests/SobolSamplerTests.swift:9-140   Sobol utilities, sample ranges
  Tests/libgonzalesTests/BoundsTests.swift:26-180        surface area, extent, slab tests
  Sobol direction numbers: the first columns of dimensions 1 and 2 are the
  classical Sobol values (Joe & Kuo 2008).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import pyoracle as O

L = O.lib


# --------------------------------------------------------- SobolSamplerTests.swift

def test_reverse_bits32_kats():
    assert L().orc_reverse_bits32(0) == 0
    assert L().orc_reverse_bits32(0xFFFFFFFF) == 0xFFFFFFFF
    assert L().orc_reverse_bits32(0x80000000) == 1
    for v in [0, 1, 42, 0xDEADBEEF, 0x12345678, 0xFFFFFFFF]:
        assert L().orc_reverse_bits32(L().orc_reverse_bits32(v)) == v


def test_encode_morton2_kats():
    assert L().orc_encode_morton2(0, 0) == 0
    assert L().orc_encode_morton2(1, 0) == 1
    assert L().orc_encode_morton2(0, 1) == 2
    assert L().orc_encode_morton2(1, 1) == 3


def test_mix_bits_kats():
    assert L().orc_mix_bits(12345) == L().orc_mix_bits(12345)
    a, b, c = L().orc_mix_bits(0), L().orc_mix_bits(1), L().orc_mix_bits(99999)
    assert a != b and a != c and b != c


def test_next_power_of_two_kats():
    for v, e in [(16, 16), (1, 1), (1024, 1024), (3, 4), (5, 8), (17, 32), (100, 128)]:
        assert L().orc_next_power_of_two(v) == e


def test_owen_scrambler_kats():
    assert L().orc_owen_scramble(12345, 42) == L().orc_owen_scramble(12345, 42)
    assert L().orc_owen_scramble(12345, 1) != L().orc_owen_scramble(12345, 2)


@pytest.mark.parametrize("kind,pixel,count", [(1, (10, 10), 20), (2, (5, 5), 10), (3, (5, 5), 10)])
def test_zsobol_values_in_range(kind, pixel, count):
    # SobolSamplerTests.swift:96-140: spp 4, 64x64, seed 0.
    out = O.zsobol_batch(4, 64, 64, [pixel[0]], [pixel[1]], [0], [kind] * count, seed=0)
    assert out.shape == (1, kind * count)
    assert (out >= 0).all() and (out < 1).all()


# --------------------------------------------------------- Sobol matrices

def test_sobol_matrix_first_columns():
    m = np.fromfile(O.SOBOL, dtype="<u4").reshape(1024, 52)
    assert [int(x) for x in m[0, :32]] == [1 << (31 - i) for i in range(32)]
    assert not m[0, 32:].any()
    # dimension 1: Pascal's triangle mod 2 (classical second Sobol dimension)
    assert [hex(int(x)) for x in m[1, :6]] == ["0x80000000", "0xc0000000", "0xa0000000", "0xf0000000",
                                               "0x88000000", "0xcc000000"]
    # dimension 2: s=2, a=1, m=(1,3)
    assert [hex(int(x)) for x in m[2, :4]] == ["0x80000000", "0xc0000000", "0x60000000", "0x90000000"]


def test_sobol_sample_unscrambled_is_van_der_corput():
    # With the scrambler seed forced through reverse/hash this is not directly
    # observable, so check the matrix product itself: index i in dim 0 gives
    # bit-reversed i.
    m = np.fromfile(O.SOBOL, dtype="<u4").reshape(1024, 52)
    for i in [1, 2, 3, 5, 77, 1023]:
        acc = 0
        for b in range(52):
            if (i >> b) & 1:
                acc ^= int(m[0, b])
        assert acc == L().orc_reverse_bits32(i)


def test_zsobol_sample_index_is_permutation_within_pixel():
    # getSampleIndex permutes base-4 digits: within a pixel the 16 sample
    # indices of a 16-spp sampler map to 16 distinct indices with the pixel's
    # Morton prefix.
    st = O.ZSobolState()
    seen = set()
    for i in range(16):
        L().orc_zsobol_init(O.C.byref(st), 16, 64, 64, 1234)
        L().orc_zsobol_start_pixel_sample(O.C.byref(st), 3, 5, i, 0)
        seen.add(L().orc_zsobol_sample_index(O.C.byref(st)))
    assert len(seen) == 16
    prefix = {s >> 4 for s in seen}
    assert len(prefix) == 1


# --------------------------------------------------------- BoundsTests.swift

def test_bounds_surface_area_kats():
    assert abs(O.surface_area([0, 0, 0], [1, 1, 1]) - 6.0) <= 1e-6
    assert abs(O.surface_area([0, 0, 0], [2, 3, 4]) - 52.0) <= 1e-6


def test_bounds_maximum_extent_kats():
    assert O.maximum_extent([0, 0, 0], [10, 1, 1]) == 0
    assert O.maximum_extent([0, 0, 0], [1, 10, 1]) == 1
    assert O.maximum_extent([0, 0, 0], [1, 1, 10]) == 2


def _n(v):
    v = np.asarray(v, np.float32)
    return (v / np.sqrt(np.float32((v * v).sum()))).astype(np.float32)


SLAB_CASES = [
    # (origin, direction, tHit, expected) from BoundsTests.swift:120-180
    ((0, 0, 5), (0, 0, -1), np.inf, True),
    ((0, 5, 0), _n((0.01, 1, 0.01)), np.inf, False),
    ((0, 0, 5), _n((0.001, 0.001, 1)), np.inf, False),
    ((0, 0, 5), _n((0.001, 0.001, -1)), 3.0, False),
    ((0, 0, 5), _n((0.001, 0.001, -1)), 10.0, True),
    ((0, 0, 0), (1, 0, 0), np.inf, True),
    ((-5, -5, -5), _n((1, 1, 1)), np.inf, True),
]


@pytest.mark.parametrize("o,d,thit,expected", SLAB_CASES)
def test_swift_slab_kats(o, d, thit, expected):
    assert O.bounds_intersects_swift([-1, -1, -1], [1, 1, 1], o, d, thit) == expected


@pytest.mark.parametrize("o,d,thit,expected", SLAB_CASES)
def test_reference_kernel_slab_on_kats(o, d, thit, expected):
    # The Mojo slab test (kernel.mojo:171-206) precomputes org * (1/dir); for a
    # direction component of +-0 with a zero origin component that is 0 * inf =
    # NaN, every comparison with it is false and the box is culled.  On the
    # Swift test's cases it therefore agrees except where that happens.
    hit, _ = O.aabb([-1, -1, -1], [1, 1, 1], o, d, thit)
    nan_axis = any(float(oi) == 0.0 and float(di) == 0.0 for oi, di in zip(o, d))
    assert hit == (expected and not nan_axis)


# --------------------------------------------------------- leaf tests

def test_mt_known_answers():
    p0, p1, p2 = [0, 0, 0], [1, 0, 0], [0, 1, 0]
    hit, t, u, v = O.mt([0.25, 0.25, 1], [0, 0, -1], p0, p1, p2, np.inf)
    assert hit and t == 1.0 and u == 0.25 and v == 0.25
    assert not O.mt([0.25, 0.25, 1], [0, 0, -1], p0, p1, p2, 0.5)[0]      # beyond tMax
    assert O.mt([0.25, 0.25, 1], [0, 0, -1], p0, p1, p2, 1.0)[0]          # t == tMax accepted
    assert not O.mt([0.25, 0.25, -1], [0, 0, -1], p0, p1, p2, np.inf)[0]  # behind origin
    assert not O.mt([0.8, 0.8, 1], [0, 0, -1], p0, p1, p2, np.inf)[0]     # outside
    assert not O.mt([0, 0, 1], [1, 0, 0], p0, p1, p2, np.inf)[0]          # parallel: |det| < 1e-7


def test_watertight_known_answers():
    p0, p1, p2 = [0, 0, 0], [1, 0, 0], [0, 1, 0]
    hit, t, b0, b1, b2 = O.watertight([0.25, 0.25, 1], [0, 0, -1], p0, p1, p2, np.inf)
    assert hit and t == 1.0 and (b0, b1, b2) == (0.5, 0.25, 0.25)
    # a ray through the shared edge of two triangles hits at least one of them
    q0, q1, q2 = [1, 0, 0], [1, 1, 0], [0, 1, 0]
    o, d = [0.5, 0.5, 1], [0, 0, -1]
    assert O.watertight(o, d, p0, p1, p2, np.inf)[0] or O.watertight(o, d, q0, q1, q2, np.inf)[0]


# --------------------------------------------------------- committed fixtures

def test_oracle_reproduces_golden_raycast():
    from gonzales_b200 import scenes

    g = np.load(Path(__file__).resolve().parent / "golden" / "raycast_small.npz")
    hs = scenes.raycast_scene(subdiv=int(g["subdiv"])).build()
    assert hs.nodes.tobytes() == g["nodes"].tobytes()
    r6 = scenes.pack_reference_rays(g["o"], g["d"])
    isect, idx, _ = O.traverse(hs.nodes, hs.prims, [(m.points, m.vertex_indices) for m in hs.meshes], r6, g["t"])
    assert np.array_equal(idx, g["prim"])
    assert isect["t_hit"].tobytes() == g["t_hit"].tobytes()
    assert 0.2 < (idx >= 0).mean() < 1.0


def test_oracle_reproduces_golden_zsobol():
    g = np.load(Path(__file__).resolve().parent / "golden" / "zsobol_small.npz")
    vals = O.zsobol_batch(16, 256, 256, g["px"], g["py"], g["index"], g["kinds"], seed=1234)
    assert vals.tobytes() == g["values"].tobytes()
    assert (vals >= 0).all() and (vals < 1).all()
