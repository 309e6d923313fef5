"""Minimal PNG writer for displayed images (8-bit RGBA, no external imaging library)."""
import struct
import zlib

import numpy as np


def png_bytes(rgba):
    """PNG file contents of an (H, W, 4) uint8 array whose row 0 is the top row."""
    a = np.ascontiguousarray(rgba, np.uint8)
    h, w, c = a.shape
    if c != 4:
        raise ValueError("expected RGBA")
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))  # filter type 0 per scanline

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


def write_png(path, rgba):
    with open(path, "wb") as f:
        f.write(png_bytes(rgba))
