"""Image output of the headless renderer (Engine.render): linear RGBA in
[0, 1] -> 8-bit sRGB, written as binary PPM (P6).  The reference's render
target is BGRA8Unorm_sRGB, which stores linear colour with this encoding."""
from __future__ import annotations

import numpy as np


def to_srgb8(rgba) -> np.ndarray:
    """(H, W, 4) linear float -> (H, W, 3) uint8 sRGB (IEC 61966-2-1 curve)."""
    if hasattr(rgba, "detach"):
        rgba = rgba.detach().cpu().numpy()
    c = np.clip(np.asarray(rgba, np.float64)[..., :3], 0.0, 1.0)
    s = np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(c, 1.0 / 2.4) - 0.055)
    return np.round(s * 255.0).astype(np.uint8)


def write_ppm(path: str, rgba) -> None:
    img = to_srgb8(rgba)
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(img.tobytes())


def write_png(path: str, rgba) -> None:
    """8-bit sRGB PNG (RGB, no filtering), standard library only."""
    import struct
    import zlib

    img = to_srgb8(rgba)
    h, w = img.shape[:2]
    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))
