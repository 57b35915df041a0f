"""Headless projection images: the RGBA buffers of bec_render_projections written as
24-bit BMP files (the reference's createBitmap, programs/bec_wigner_3d.cuda/bitmap.h:90-144,
writes its zy projection the same way; it reads the colours back from an OpenGL buffer).
"""
import struct

import numpy as np


def write_bmp(path, rgba):
    """rgba: (h, w, 4) floats in [0, 1]; row 0 is the top of the image."""
    img = np.clip(np.asarray(rgba)[..., :3] * 256.0, 0, 255).astype(np.uint8)
    h, w = img.shape[:2]
    row = (3 * w + 3) // 4 * 4
    size = 54 + row * h
    with open(path, "wb") as f:
        f.write(struct.pack("<2sIHHI", b"BM", size, 0, 0, 54))
        f.write(struct.pack("<IiiHHIIiiII", 40, w, h, 1, 24, 0, row * h, 2835, 2835, 0, 0))
        pad = b"\0" * (row - 3 * w)
        for y in range(h - 1, -1, -1):          # bottom-up rows, BGR
            f.write(img[y, :, ::-1].tobytes() + pad)


def read_bmp(path):
    """(h, w, 3) uint8 RGB of a 24-bit BMP written by write_bmp."""
    with open(path, "rb") as f:
        data = f.read()
    off = struct.unpack_from("<I", data, 10)[0]
    w, h = struct.unpack_from("<ii", data, 18)
    row = (3 * w + 3) // 4 * 4
    out = np.zeros((h, w, 3), dtype=np.uint8)
    for y in range(h):
        line = np.frombuffer(data, dtype=np.uint8, count=3 * w, offset=off + (h - 1 - y) * row)
        out[y] = line.reshape(w, 3)[:, ::-1]
    return out


def ramp(u):
    """The blue-white-yellow-red ramp of spectre.cu:34-46 (765 texels, linear filtering,
    clamped), evaluated for levels u = level / max; returns (..., 3) floats."""
    u = np.clip(np.asarray(u, dtype=np.float64), 0.0, 1.0)
    p = u * 765 - 0.5
    i0 = np.floor(p).astype(int)
    f = p - i0
    i1 = np.clip(i0 + 1, 0, 764)
    i0 = np.clip(i0, 0, 764)

    def tex(i):
        r = np.where(i <= 255, i, 255)
        g = np.where(i <= 255, i, np.where(i <= 510, 255, 765 - i))
        b = np.where(i <= 255, 255, np.where(i <= 510, 510 - i, 0))
        return np.stack([r, g, b], axis=-1) / 256.0

    c0, c1 = tex(i0), tex(i1)
    return c0 + f[..., None] * (c1 - c0)


def save_projections(eng, group, prefix):
    """Writes <prefix>_{xy,zy}_{a,b}.bmp for one group of an Engine; returns the file names."""
    img = eng.render_projections(group)
    names = []
    for k in ("xy_a", "xy_b", "zy_a", "zy_b"):
        n = f"{prefix}_{k}.bmp"
        write_bmp(n, img[k])
        names.append(n)
    return names
