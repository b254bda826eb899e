"""Writes the committed golden fixtures from the oracle (the CPU restatement of
the reference path).  Re-run after an intentional oracle change:

    python tests/golden/make_golden.py

raycast_small.npz: displaced icosphere (subdiv 3), 1024 coherent + 1024
    incoherent rays, BVH2 nodes, closest-hit prim index / t / u / v.
zsobol_small.npz: Z-Sobol values (seed 1234) for 64 pixel samples of a
    256x256, 16-spp sampler, drawing get2D, get2D, then get1D/get2D/get3D
    repeatedly (the dimension pattern of a camera sample plus bounces).
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gonzales_b200 import scenes  # noqa: E402
from oracle import pyoracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def raycast_small():
    subdiv = 3
    hs = scenes.raycast_scene(subdiv=subdiv).build()
    o, d, t = scenes.raycast_rays(hs, 32, 32, 1024, seed=0x60)
    r6 = scenes.pack_reference_rays(o, d)
    isect, idx, _ = O.traverse(hs.nodes, hs.prims, [(m.points, m.vertex_indices) for m in hs.meshes], r6, t)
    np.savez_compressed(OUT / "raycast_small.npz", subdiv=subdiv, nodes=hs.nodes, o=o, d=d, t=t, prim=idx,
                        t_hit=isect["t_hit"], u=isect["u"], v=isect["v"])


ZSOBOL_KINDS = [2, 2] + [1, 2, 3, 2] * 6


def zsobol_small():
    rng = np.random.default_rng(5)
    px = rng.integers(0, 256, 64)
    py = rng.integers(0, 256, 64)
    idx = rng.integers(0, 16, 64)
    vals = O.zsobol_batch(16, 256, 256, px, py, idx, ZSOBOL_KINDS, seed=1234)
    np.savez_compressed(OUT / "zsobol_small.npz", px=px, py=py, index=idx, kinds=np.array(ZSOBOL_KINDS),
                        values=vals)


if __name__ == "__main__":
    raycast_small()
    zsobol_small()
    print("golden fixtures written to", OUT)
