"""Shared test helpers: scene construction and the parity classifier.

Parity rule (per ray, GPU vs oracle closest hit):
  exact            same prim, t/u/v bit-identical (or both miss)
  tie              different prim, same t bits, GPU prim is a valid MT hit at that t
                   (equal-t triangles resolved in a different visit order)
  reference-culled GPU t < oracle t (or oracle missed) and the GPU's triangle is
                   a valid MT hit with exactly the GPU's t/u/v: the reference's
                   non-conservative slab test (kernel.mojo:204) culled a node
  fail             anything else (in particular the GPU missing a hit or
                   returning a farther one)
"""
import json
import os
from pathlib import Path

import numpy as np

from gonzales_b200 import scenes
from oracle import pyoracle as O


def mesh_list(hs):
    return [(m.points, m.vertex_indices) for m in hs.meshes]


def prim_triangle(hs, k):
    p = hs.prims[k]
    if p["type"] == 0:
        mesh, base = int(p["id1"]), int(p["id2"])
    else:
        mesh, base = int(p["id2"]) >> 32, (int(p["id2"]) & 0xFFFFFFFF) * 3
    m = hs.meshes[mesh]
    idx = m.vertex_indices[base:base + 3]
    return [m.points[i, :3] for i in idx]


def oracle_closest(hs, o, d, t, watertight=False):
    r6 = scenes.pack_reference_rays(o, d)
    return O.traverse(hs.nodes, hs.prims, mesh_list(hs), r6, t, watertight=watertight)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def classify(hs, o, d, tmax, gpu_prim, gpu_t, gpu_u, gpu_v, ora_idx, ora_t, ora_u, ora_v, watertight=False):
    """Returns dict of counts and the indices of failures."""
    gpu_prim = np.asarray(gpu_prim, np.int64)
    ora_idx = np.asarray(ora_idx, np.int64)
    same = (gpu_prim == ora_idx)
    both_hit = same & (ora_idx >= 0)
    exact = (same & (ora_idx < 0)) | (both_hit & (bits(gpu_t) == bits(ora_t)) & (bits(gpu_u) == bits(ora_u))
                                      & (bits(gpu_v) == bits(ora_v)))
    counts = {"rays": len(gpu_prim), "exact": int(exact.sum()), "tie": 0, "reference_culled": 0, "fail": 0}
    fails = []
    for i in np.nonzero(~exact)[0]:
        g = int(gpu_prim[i])
        if g < 0:
            fails.append(i)
            continue
        p0, p1, p2 = prim_triangle(hs, g)
        if watertight:
            ok, t, b0, b1, b2 = O.watertight(o[i], d[i], p0, p1, p2, float(tmax[i]))
            u, v = b1, b2
        else:
            ok, t, u, v = O.mt(o[i], d[i], p0, p1, p2, float(tmax[i]))
        valid = ok and bits(t) == bits(gpu_t[i]) and bits(u) == bits(gpu_u[i]) and bits(v) == bits(gpu_v[i])
        if not valid:
            fails.append(i)
        elif ora_idx[i] >= 0 and bits(gpu_t[i]) == bits(ora_t[i]):
            counts["tie"] += 1
        elif ora_idx[i] < 0 or gpu_t[i] < ora_t[i]:
            counts["reference_culled"] += 1
        else:
            fails.append(i)
    counts["fail"] = len(fails)
    return counts, fails


def small_raycast(subdiv=4, n_side=48, n_incoherent=4096, seed=0xC1):
    sb = scenes.raycast_scene(subdiv=subdiv, seed=seed)
    hs = sb.build()
    o, d, t = scenes.raycast_rays(hs, n_side, n_side, n_incoherent, seed=seed)
    return hs, o, d, t


def record(name, data):
    """Writes a measurement record (JSON) into $GZG_RECORD_DIR when it is set."""
    d = os.environ.get("GZG_RECORD_DIR")
    if d and Path(d).is_dir():
        (Path(d) / name).write_text(json.dumps(data))
