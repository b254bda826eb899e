"""Builds tests/golden/regression_test.npz from the reference's render
regression test: the scene Tests/reference/regression-test.pbrt and its golden
image Tests/reference/regression-test.exr (with albedo.exr and normal.exr
beside it).  The reference test (Tests/libgonzalesTests/RenderRegressionTests
.swift:9-72) renders the scene and requires a normalised RMSE below 0.1
against the golden image.

Usage (in a tree where the Gonzales sources are present):

    python tests/golden/make_regression_golden.py /path/to/Gonzales

The fixture holds the scene as plain arrays (per mesh: points, indices,
vertex normals, UVs and its named material's reflectance; the area light's
radiance; camera transform, fov, film size, samples per pixel, maximum depth
and Gaussian filter) and the three decoded images as float32 (H, W, 4) RGBA.

Only what this scene uses is parsed: Integrator, Transform, Sampler,
PixelFilter, Film, Camera, MakeNamedMaterial (diffuse reflectance),
NamedMaterial, Shape "trianglemesh", AreaLightSource "diffuse" and
AttributeBegin/End.  The EXR reader handles single-part, one-level tiled or
scanline files with FLOAT or HALF channels and NONE, ZIPS or ZIP compression
(the OpenEXR file layout: magic, header attributes, chunk offset table,
chunks; ZIP chunks are zlib streams of byte-split, delta-coded data).
"""
import re
import struct
import sys
import zlib
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "regression_test.npz"


# ---------------------------------------------------------------- PBRT

def _tokens(text):
    text = re.sub(r"#[^\n]*", "", text)
    return re.findall(r'"[^"]*"|\[|\]|[^\s\[\]"]+', text)


def _params(toks, i):
    """Parses '"type name" value' pairs from toks[i:]; returns (dict, next i)."""
    out = {}
    while i < len(toks) and toks[i].startswith('"') and len(toks[i][1:-1].split()) == 2:
        typ, name = toks[i][1:-1].split()
        i += 1
        if toks[i] == "[":
            j = toks.index("]", i)
            vals = toks[i + 1:j]
            i = j + 1
        else:
            vals = [toks[i]]
            i += 1
        if typ in ("string", "texture", "bool"):
            out[name] = [v.strip('"') for v in vals]
        elif typ == "integer":
            out[name] = [int(v) for v in vals]
        else:
            out[name] = [float(v) for v in vals]
    return out, i


def parse_pbrt(path):
    toks = _tokens(Path(path).read_text())
    scene = {"meshes": [], "materials": {}}
    current_material = None
    area_light = None
    stack = []
    i = 0
    while i < len(toks):
        t = toks[i]
        i += 1
        if t == "Transform":
            j = toks.index("]", i)
            scene["transform"] = np.array([float(v) for v in toks[i + 1:j]], np.float64)
            i = j + 1
        elif t in ("Integrator", "Sampler", "PixelFilter", "Film", "Camera", "Accelerator"):
            kind = toks[i].strip('"')
            params, i = _params(toks, i + 1)
            scene[t.lower()] = (kind, params)
        elif t == "WorldBegin":
            pass
        elif t == "MakeNamedMaterial":
            name = toks[i].strip('"')
            params, i = _params(toks, i + 1)
            scene["materials"][name] = params
        elif t == "NamedMaterial":
            current_material = toks[i].strip('"')
            i += 1
        elif t == "AttributeBegin":
            stack.append((current_material, area_light))
        elif t == "AttributeEnd":
            current_material, area_light = stack.pop()
        elif t == "AreaLightSource":
            kind = toks[i].strip('"')
            params, i = _params(toks, i + 1)
            assert kind == "diffuse", kind
            area_light = params["L"]
        elif t == "Shape":
            kind = toks[i].strip('"')
            params, i = _params(toks, i + 1)
            assert kind == "trianglemesh", kind
            scene["meshes"].append({"material": current_material, "L": area_light, "P": params["P"],
                                    "indices": params["indices"], "N": params.get("N"), "uv": params.get("uv")})
        else:
            raise ValueError("unexpected token %r" % t)
    return scene


# ---------------------------------------------------------------- OpenEXR

def _attributes(b, p):
    hdr = {}
    while True:
        e = b.index(b"\0", p)
        name = b[p:e].decode()
        p = e + 1
        if not name:
            return hdr, p
        e = b.index(b"\0", p)
        typ = b[p:e].decode()
        p = e + 1
        size = struct.unpack_from("<i", b, p)[0]
        p += 4
        hdr[name] = (typ, b[p:p + size])
        p += size


def _channels(raw):
    out, p = [], 0
    while raw[p] != 0:
        e = raw.index(b"\0", p)
        name = raw[p:e].decode()
        ptype, _, xs, ys = struct.unpack_from("<iB3xii", raw, e + 1)
        assert xs == 1 and ys == 1
        out.append((name, ptype))
        p = e + 1 + 16
    return out


def _unzip(data, expected):
    t = np.frombuffer(zlib.decompress(data), np.uint8)
    assert len(t) == expected, (len(t), expected)
    # undo the predictor (each byte stored as the difference to the previous
    # one, plus 128), then re-interleave the two halves
    d = t.astype(np.int64)
    d[1:] -= 128
    t = (np.cumsum(d) & 0xFF).astype(np.uint8)
    half = (len(t) + 1) // 2
    out = np.empty_like(t)
    out[0::2] = t[:half]
    out[1::2] = t[half:]
    return out.tobytes()


def read_exr(path):
    """(H, W, C) float32 array with channels in R, G, B, A order (those present)."""
    b = Path(path).read_bytes()
    assert b[:4] == b"\x76\x2f\x31\x01", "not an OpenEXR file"
    flags = struct.unpack_from("<I", b, 4)[0]
    tiled = bool(flags & 0x200)
    assert not flags & 0x1800, "deep or multi-part files are not read"
    hdr, p = _attributes(b, 8)
    chans = _channels(hdr["channels"][1])
    comp = hdr["compression"][1][0]
    assert comp in (0, 2, 3), "compression %d not read" % comp
    x0, y0, x1, y1 = struct.unpack("<4i", hdr["dataWindow"][1])
    W, H = x1 - x0 + 1, y1 - y0 + 1
    size = {1: 2, 2: 4}
    dt = {1: "<f2", 2: "<f4"}
    img = {name: np.zeros((H, W), np.float32) for name, _ in chans}
    if tiled:
        tx, ty, mode = struct.unpack("<IIB", hdr["tiles"][1])
        assert mode & 0xF == 0, "mip levels are not read"
        ntx, nty = -(-W // tx), -(-H // ty)
        offsets = struct.unpack_from("<%dQ" % (ntx * nty), b, p)
        for off in offsets:
            cx, cy, lx, ly, n = struct.unpack_from("<5i", b, off)
            assert lx == 0 and ly == 0
            data = b[off + 20:off + 20 + n]
            w = min(tx, W - cx * tx)
            h = min(ty, H - cy * ty)
            expected = h * w * sum(size[t] for _, t in chans)
            raw = data if (comp == 0 or n == expected) else _unzip(data, expected)
            q = 0
            for r in range(h):
                for name, t in chans:
                    nb = w * size[t]
                    img[name][cy * ty + r, cx * tx:cx * tx + w] = np.frombuffer(raw[q:q + nb], dt[t])
                    q += nb
    else:
        lines = {0: 1, 2: 1, 3: 16}[comp]
        nchunks = -(-H // lines)
        offsets = struct.unpack_from("<%dQ" % nchunks, b, p)
        for off in offsets:
            yy, n = struct.unpack_from("<2i", b, off)
            data = b[off + 8:off + 8 + n]
            h = min(lines, y1 + 1 - yy)
            expected = h * W * sum(size[t] for _, t in chans)
            raw = data if (comp == 0 or n == expected) else _unzip(data, expected)
            q = 0
            for r in range(h):
                for name, t in chans:
                    nb = W * size[t]
                    img[name][yy - y0 + r] = np.frombuffer(raw[q:q + nb], dt[t])
                    q += nb
    order = [c for c in "RGBA" if c in img]
    return np.stack([img[c] for c in order], -1)


def main(root):
    root = Path(root)
    ref = root / "Tests" / "reference"
    sc = parse_pbrt(ref / "regression-test.pbrt")
    arrays = {}
    names = []
    for k, m in enumerate(sc["meshes"]):
        arrays["mesh%d_P" % k] = np.asarray(m["P"], np.float32).reshape(-1, 3)
        arrays["mesh%d_indices" % k] = np.asarray(m["indices"], np.int64)
        arrays["mesh%d_N" % k] = np.asarray(m["N"], np.float32).reshape(-1, 3)
        arrays["mesh%d_uv" % k] = np.asarray(m["uv"], np.float32).reshape(-1, 2)
        mat = sc["materials"][m["material"]]
        arrays["mesh%d_reflectance" % k] = np.asarray(mat["reflectance"], np.float32)
        arrays["mesh%d_L" % k] = np.asarray(m["L"] if m["L"] is not None else [0, 0, 0], np.float32)
        names.append(m["material"])
    arrays["mesh_materials"] = np.array(names)
    arrays["camera_transform"] = sc["transform"].astype(np.float64)
    arrays["fov"] = np.float64(sc["camera"][1]["fov"][0])
    film = sc["film"][1]
    arrays["resolution"] = np.array([film["xresolution"][0], film["yresolution"][0]], np.int64)
    arrays["spp"] = np.int64(sc["sampler"][1]["pixelsamples"][0])
    arrays["sampler"] = np.array(sc["sampler"][0])
    arrays["max_depth"] = np.int64(sc["integrator"][1]["maxdepth"][0])
    pf = sc["pixelfilter"][1]
    arrays["filter_radius"] = np.array([pf["xradius"][0], pf["yradius"][0]], np.float64)
    arrays["filter_sigma"] = np.float64(pf["sigma"][0])
    arrays["golden"] = read_exr(ref / "regression-test.exr")
    arrays["golden_albedo"] = read_exr(ref / "albedo.exr")
    arrays["golden_normal"] = read_exr(ref / "normal.exr")
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT, "meshes", len(names), "image", arrays["golden"].shape)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
