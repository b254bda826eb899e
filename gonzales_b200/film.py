"""Film output: normalising the device film sums (gzg_film_resolve_device,
Pixel.normalized of Core/Pixel.swift) and OpenEXR files (gzg_write_exr, the
RGBA float images Image/OpenImageIOWriter.swift writes)."""
import ctypes as C
import struct

import numpy as np

from . import _ffi as F


def resolve(film_rgb, film_w, stream=None):
    """image = film_rgb / film_w (torch CUDA tensors (..., 3) and (...)), black
    stays black; returns (image, number of non-black pixels with weight 0)."""
    import torch

    n = film_w.numel()
    image = torch.empty_like(film_rgb)
    zero = torch.zeros(1, dtype=torch.int64, device=film_rgb.device)
    F.check(F.lib().gzg_film_resolve_device(film_rgb.data_ptr(), film_w.data_ptr(), n, image.data_ptr(),
                                            zero.data_ptr(), stream.cuda_stream if stream is not None else None))
    return image, int(zero.item())


def write_exr(path, image):
    """Writes (height, width, 3 or 4) float32 as an RGBA float OpenEXR file."""
    image = np.ascontiguousarray(image, np.float32)
    h, w, c = image.shape
    F.check(F.lib().gzg_write_exr(str(path).encode(), F.ptr(image), w, h, c))


def read_exr(path):
    """Reads an uncompressed single-part scanline OpenEXR file with FLOAT
    channels (what write_exr writes) into (height, width, channels) float32,
    channels in R, G, B, A order when present; returns (image, header dict)."""
    data = open(path, "rb").read()
    if struct.unpack_from("<I", data, 0)[0] != 20000630:
        raise ValueError("not an OpenEXR file")
    version = struct.unpack_from("<I", data, 4)[0]
    if version & 0xFF != 2 or version & ~0xFF:
        raise ValueError("only single-part scanline version 2 files are read")
    pos = 8
    header = {}

    def cstr(p):
        e = data.index(b"\0", p)
        return data[p:e].decode(), e + 1

    while data[pos] != 0:
        name, pos = cstr(pos)
        typ, pos = cstr(pos)
        size = struct.unpack_from("<I", data, pos)[0]
        pos += 4
        header[name] = (typ, data[pos:pos + size])
        pos += size
    pos += 1
    chans = []
    raw = header["channels"][1]
    p = 0
    while raw[p] != 0:
        e = raw.index(b"\0", p)
        nm = raw[p:e].decode()
        ptype = struct.unpack_from("<i", raw, e + 1)[0]
        chans.append((nm, ptype))
        p = e + 1 + 16
    if any(t != 2 for _, t in chans):
        raise ValueError("only FLOAT channels are read")
    if header["compression"][1] != b"\x00":
        raise ValueError("only uncompressed files are read")
    x0, y0, x1, y1 = struct.unpack("<4i", header["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack_from("<%dQ" % h, data, pos)
    img = np.zeros((h, w, len(chans)), np.float32)
    for off in offsets:
        y, nbytes = struct.unpack_from("<iI", data, off)
        line = np.frombuffer(data, np.float32, nbytes // 4, off + 8).reshape(len(chans), w)
        img[y - y0] = line.T
    names = [n for n, _ in chans]
    order = [names.index(n) for n in ("R", "G", "B", "A") if n in names]
    return img[..., order], {k: v[0] for k, v in header.items()}


__all__ = ["resolve", "write_exr", "read_exr"]
