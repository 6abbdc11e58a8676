"""Image files on either side of the render: Radiance RGBE (.hdr) read and
write, 8-bit PNG write, and the tone maps the reference offers.

Follows dort.image (src/dort/lua_image.cpp, image.cpp:14-66): RGBE is
written with the encoder of the reference's stb_image_write (per pixel the
shared exponent of the largest channel, mantissas truncated to 8 bits, flat
scanlines) and read with the usual decoding value = m * 2^(e - 136) (RLE or
flat scanlines); PNG is 8-bit RGB of a tone-mapped image.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np


def rgbe_encode(img) -> np.ndarray:
    """float RGB [h, w, 3] -> uint8 RGBE [h, w, 4] (truncating mantissas)."""
    img = np.asarray(img, np.float32)
    mx = img.max(axis=-1)
    out = np.zeros(img.shape[:-1] + (4,), np.uint8)
    ok = mx >= 1e-32
    m, e = np.frexp(mx[ok])
    norm = (m * 256.0 / mx[ok]).astype(np.float32)
    vals = img[ok] * norm[:, None]
    out[ok, :3] = np.clip(vals, 0, 255).astype(np.uint8)   # C cast truncates
    out[ok, 3] = (e + 128).astype(np.uint8)
    return out


def rgbe_decode(rgbe) -> np.ndarray:
    """uint8 RGBE [h, w, 4] -> float RGB [h, w, 3]."""
    rgbe = np.asarray(rgbe, np.uint8)
    e = rgbe[..., 3].astype(np.int32)
    f = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0).astype(np.float32)
    return rgbe[..., :3].astype(np.float32) * f[..., None]


def rgbe_quantize(img) -> np.ndarray:
    """The values an image has after a write to and read from an RGBE file."""
    return rgbe_decode(rgbe_encode(img))


def write_rgbe(path: str, img) -> None:
    img = np.asarray(img, np.float32)
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\n# Written by dort_b200\nFORMAT=32-bit_rle_rgbe\n\n")
        f.write(b"-Y %d +X %d\n" % (h, w))
        f.write(rgbe_encode(img).tobytes())


def read_rgbe(path: str) -> np.ndarray:
    """Radiance .hdr (flat or new-style RLE scanlines) -> float RGB [h, w, 3]."""
    data = open(path, "rb").read()
    pos = 0
    h = w = None
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end]
        pos = end + 1
        if line.startswith(b"-Y ") or line.startswith(b"+Y "):
            parts = line.split()
            if parts[0] != b"-Y" or parts[2] != b"+X":
                raise ValueError(f"unsupported orientation {line!r}")
            h, w = int(parts[1]), int(parts[3])
            break
    img = np.zeros((h, w, 4), np.uint8)
    for y in range(h):
        rle = (w >= 8 and w < 32768 and data[pos] == 2 and data[pos + 1] == 2
               and (data[pos + 2] & 0x80) == 0)
        if rle:
            if (data[pos + 2] << 8 | data[pos + 3]) != w:
                raise ValueError("bad scanline width")
            pos += 4
            for c in range(4):
                x = 0
                while x < w:
                    n = data[pos]
                    pos += 1
                    if n > 128:
                        n -= 128
                        img[y, x:x + n, c] = data[pos]
                        pos += 1
                    else:
                        img[y, x:x + n, c] = np.frombuffer(data, np.uint8, n, pos)
                        pos += n
                    x += n
        else:
            img[y] = np.frombuffer(data, np.uint8, 4 * w, pos).reshape(w, 4)
            pos += 4 * w
    return rgbe_decode(img)


def tonemap_srgb(img) -> np.ndarray:
    """Linear RGB -> sRGB-encoded values in [0, 1]."""
    x = np.clip(np.asarray(img, np.float64), 0.0, 1.0)
    return np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x, 1 / 2.4) - 0.055)


def tonemap_gamma(img, gamma: float = 2.2) -> np.ndarray:
    return np.power(np.clip(np.asarray(img, np.float64), 0.0, 1.0), 1.0 / gamma)


def write_png(path: str, img) -> None:
    """8-bit RGB PNG of values in [0, 1] (tone-map first)."""
    a = np.clip(np.rint(np.asarray(img, np.float64) * 255.0), 0, 255).astype(np.uint8)
    h, w = a.shape[:2]
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))

    def chunk(tag, payload):
        return (struct.pack(">I", len(payload)) + tag + payload
                + struct.pack(">I", zlib.crc32(tag + payload) & 0xFFFFFFFF))

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def write_pfm(path: str, img) -> None:
    """Portable float map (little-endian, bottom row first): signed float RGB,
    the format the Lua front-end's dort.image.write_pfm writes."""
    a = np.asarray(img, np.float32)
    h, w = a.shape[:2]
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1.0\n" % (w, h))
        f.write(np.ascontiguousarray(a[::-1]).astype("<f4").tobytes())


def read_pfm(path: str) -> np.ndarray:
    """Portable float map -> float RGB [h, w, 3] (row 0 at the top)."""
    data = open(path, "rb").read()
    lines, pos = [], 0
    while len(lines) < 3:
        end = data.index(b"\n", pos)
        lines.append(data[pos:end].strip())
        pos = end + 1
    if lines[0] != b"PF":
        raise ValueError(f"{path}: not an RGB portable float map")
    w, h = (int(x) for x in lines[1].split())
    scale = float(lines[2])
    dt = "<f4" if scale < 0 else ">f4"
    a = np.frombuffer(data, dt, 3 * w * h, pos).reshape(h, w, 3)
    return a[::-1].astype(np.float32)
