"""Minimal PNG reader and writer (8-bit, non-interlaced; no external imaging library): displayed
images, environment maps and the SDF-PNG assets of the reference's packer."""
import struct
import zlib

import numpy as np

_SIG = b"\x89PNG\r\n\x1a\n"
_CHANNELS = {0: 1, 2: 3, 4: 2, 6: 4}  # grey, RGB, grey + alpha, RGBA


def png_bytes(pixels):
    """PNG file contents of an (H, W, 3) or (H, W, 4) uint8 array whose row 0 is the top row."""
    a = np.ascontiguousarray(pixels, np.uint8)
    h, w, c = a.shape
    if c not in (3, 4):
        raise ValueError("expected RGB or RGBA")
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))  # filter type 0 per scanline

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    ctype = 6 if c == 4 else 2
    return (_SIG + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


def write_png(path, pixels):
    with open(path, "wb") as f:
        f.write(png_bytes(pixels))


def decode_png(data):
    """(H, W, C) uint8 array (row 0 = top row) of an 8-bit, non-interlaced PNG in grey, grey +
    alpha, RGB or RGBA (the scanline filters are undone by snelly_png_unfilter)."""
    import ctypes

    from . import _native as N
    if data[:8] != _SIG:
        raise ValueError("not a PNG file")
    pos, idat, hdr = 8, [], None
    while pos < len(data):
        n, tag = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if tag == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif tag == b"IDAT":
            idat.append(body)
        elif tag == b"IEND":
            break
    if hdr is None:
        raise ValueError("PNG without IHDR")
    w, h, depth, ctype, _, _, interlace = hdr
    if depth != 8 or ctype not in _CHANNELS or interlace != 0:
        raise ValueError("only 8-bit, non-interlaced grey/RGB(A) PNGs are supported")
    c = _CHANNELS[ctype]
    raw = zlib.decompress(b"".join(idat))
    out = np.empty((h, w, c), np.uint8)
    rc = N.lib().snelly_png_unfilter(raw, len(raw), w, h, c, out.ctypes.data)
    if rc != N.SNELLY_OK:
        raise ValueError("corrupt PNG scanlines")
    return out


def read_png(path):
    with open(path, "rb") as f:
        return decode_png(f.read())
