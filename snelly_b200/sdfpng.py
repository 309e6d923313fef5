"""The SDF-PNG asset format of the reference's packer (scripts/pngPacker.html:13-123): a signed
distance grid stored in the RGB bytes of a square PNG image, as the reference's mesh scenes load
them (exampleScenes/meshes/bunny.html:198-224) into a sampler3D.

Byte stream (RGB channels of the pixels in row order, alpha ignored): 0xBE 0xEF, version major,
version minor, metadata size (uint32 little-endian), data size (uint32 little-endian), the
metadata as UTF-8 JSON (GRES = grid resolution [x, y, z], ORIG = grid origin, EDGE = grid
extent), then the float32 samples, x fastest. The image is the smallest square holding the stream;
unused bytes are zero and alpha is 255.
"""
import json
import math
import struct

import numpy as np

from .image import decode_png, png_bytes

VERSION = (1, 0)


def pack(data, metadata):
    """PNG bytes of a float32 distance grid (any shape; flattened in C order, x fastest) and its
    metadata (a JSON-serialisable dict)."""
    md = json.dumps(metadata, separators=(",", ":")).encode("utf-8")
    samples = np.ascontiguousarray(data, np.float32).tobytes()
    raw = struct.pack("<BBBBII", 0xBE, 0xEF, VERSION[0], VERSION[1], len(md), len(samples)) + md + samples
    px = int(math.ceil(math.sqrt(len(raw) / 3.0)))
    rgb = np.zeros(px * px * 3, np.uint8)
    rgb[:len(raw)] = np.frombuffer(raw, np.uint8)
    rgba = np.full((px, px, 4), 255, np.uint8)
    rgba[..., :3] = rgb.reshape(px, px, 3)
    return png_bytes(rgba)


def unpack(png):
    """(metadata dict, float32 samples) of SDF-PNG bytes."""
    img = decode_png(png)
    if img.shape[2] < 3:
        raise ValueError("SDF-PNG needs an RGB(A) image")
    buf = np.ascontiguousarray(img[..., :3]).reshape(-1).tobytes()
    if buf[0] != 0xBE or buf[1] != 0xEF:
        raise ValueError("corrupt magic number in SDF-PNG")
    md_size, data_size = struct.unpack("<II", buf[4:12])
    if 12 + md_size + data_size > len(buf):
        raise ValueError("SDF-PNG shorter than its header states")
    metadata = json.loads(buf[12:12 + md_size].decode("utf-8"))
    data = np.frombuffer(buf[12 + md_size:12 + md_size + data_size], np.float32).copy()
    return metadata, data


def load_texture(path):
    """(metadata, sampler3D texture array of shape (GRES[2], GRES[1], GRES[0], 1) float32) of an
    SDF-PNG file, ready for shader.uniformTexture."""
    with open(path, "rb") as f:
        metadata, data = unpack(f.read())
    gx, gy, gz = (int(v) for v in metadata["GRES"])
    return metadata, data.reshape(gz, gy, gx, 1)
