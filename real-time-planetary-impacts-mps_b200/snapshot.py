"""Snapshot images as the reference writes them.

Compute::drawSnapshot (SPH/Compute/Compute.cpp:395-448) splats the material
ids into a 1024 x 1024 image (render.metal:49-66; here the CUDA kernel behind
sph_draw_snapshot) and, once the simulated time passes the next multiple of
1000 s, writes it as an RGBA PNG named snapshot_<k>.png, k = that multiple /
1000: material 402 grey (160, 160, 160), 400 orange (255, 100, 0), every
other pixel white, all opaque.  The reference encodes with lodepng; this
module writes the same pixels with its own PNG encoder (zlib, filter 0).

One difference: the reference reads the splat buffer right after encoding
the splat, before its command buffer has run, so its file holds the previous
call's image; here the file holds the image of the call that writes it.
"""
from __future__ import annotations

import os
import struct
import zlib

import numpy as np

RES = 1024
DT_MIN1 = 32.0 / 65536.0  # seconds per global-time tick (Parameters.h DT_MIN1)
_PNG_SIGNATURE = b"\x89PNG\r\n\x1a\n"


def colourise(image: np.ndarray) -> np.ndarray:
    """RGBA pixels (RES, RES, 4) uint8 of a splat image (Compute.cpp:423-439)."""
    img = np.asarray(image).reshape(RES, RES)
    out = np.full((RES, RES, 4), 255, np.uint8)
    grey = img == 402
    orange = img == 400
    out[grey, 0:3] = 160
    out[orange, 0] = 255
    out[orange, 1] = 100
    out[orange, 2] = 0
    return out


def _chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def encode_png(rgba: np.ndarray) -> bytes:
    """An 8-bit RGBA PNG of an (h, w, 4) uint8 array."""
    a = np.ascontiguousarray(rgba, np.uint8)
    if a.ndim != 3 or a.shape[2] != 4:
        raise ValueError("encode_png needs an (h, w, 4) array")
    h, w = a.shape[:2]
    rows = np.concatenate([np.zeros((h, 1), np.uint8), a.reshape(h, w * 4)], axis=1)  # filter 0 per row
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)
    return (_PNG_SIGNATURE + _chunk(b"IHDR", ihdr) + _chunk(b"IDAT", zlib.compress(rows.tobytes(), 6))
            + _chunk(b"IEND", b""))


def write_png(path: str, image: np.ndarray) -> str:
    """Colourise a splat image and write it as a PNG."""
    with open(path, "wb") as f:
        f.write(encode_png(colourise(image)))
    return path


class SnapshotWriter:
    """The reference's snapshot schedule: call after each step; when the
    simulated time exceeds the next multiple of 1000 s, splat, write
    snapshot_<k>.png into `directory` and move to the next multiple."""

    def __init__(self, directory: str = ".", every_s: int = 1000):
        self.directory = directory
        self.every_s = int(every_s)
        self.next_snapshot = 0

    def __call__(self, compute, stream=None) -> str | None:
        t = float(compute.download("global_time")[0]) * DT_MIN1
        if not t > self.next_snapshot:
            return None
        image = compute.drawSnapshot(stream)
        path = os.path.join(self.directory, f"snapshot_{self.next_snapshot // self.every_s}.png")
        write_png(path, image)
        self.next_snapshot += self.every_s
        return path
