"""Film output: OpenEXR files as SoL's Image::save writes them.

SoL saves a 3-channel film as a 32-bit float EXR whose channels are named B,
G, R and stored in that order (src/formats/exr.cpp:47-100: channel 2 of the
image first, then 1, then 0), with the writer's defaults: no compression, one
scanline per block, increasing Y.  tinyexr, which SoL uses for this, is not
available here, so the file is written directly from the OpenEXR layout
(magic number and version, attribute header, scanline offset table, scanline
blocks of per-channel rows).  `load_exr` reads back files of that form
(uncompressed, float channels).
"""
from __future__ import annotations

import struct

import numpy as np

_MAGIC = 20000630
_FLOAT = 2   # OpenEXR pixel type FLOAT


def _attr(name: str, kind: str, payload: bytes) -> bytes:
    return name.encode() + b"\0" + kind.encode() + b"\0" + struct.pack("<i", len(payload)) + payload


def save_exr(path: str, channels: np.ndarray) -> None:
    """Writes a planar film (C, H, W) float32 as SoL's exr::save does: with 3 or
    more channels, R, G, B are stored as channels named R, G, B (in the file's
    order B, G, R), a fourth as A and others as Channel_<i>."""
    ch = np.ascontiguousarray(channels, np.float32)
    if ch.ndim != 3:
        raise ValueError("channels must be (C, H, W)")
    c, h, w = ch.shape
    if c >= 3:
        order = [2, 1, 0] + list(range(3, c))
        names = ["B", "G", "R"] + (["A"] if c >= 4 else []) + [f"Channel_{i}" for i in range(4, c)]
    else:
        order = list(range(c))
        names = [f"Channel_{i}" for i in range(c)]
    chlist = b"".join(n.encode() + b"\0" + struct.pack("<iB3xii", _FLOAT, 0, 1, 1) for n in names) + b"\0"
    box = struct.pack("<iiii", 0, 0, w - 1, h - 1)
    header = (struct.pack("<ii", _MAGIC, 2)
              + _attr("channels", "chlist", chlist)
              + _attr("compression", "compression", b"\0")
              + _attr("dataWindow", "box2i", box)
              + _attr("displayWindow", "box2i", box)
              + _attr("lineOrder", "lineOrder", b"\0")
              + _attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
              + _attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
              + _attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
              + b"\0")
    row_bytes = 4 * w * c
    first = len(header) + 8 * h
    offsets = np.arange(h, dtype=np.uint64) * np.uint64(8 + row_bytes) + np.uint64(first)
    # Each block: y, byte count, then one row per channel in the file's order.
    rows = ch[order].transpose(1, 0, 2).reshape(h, c * w)            # (H, C*W)
    blocks = np.empty((h, 8 + row_bytes), np.uint8)
    blocks[:, 0:4] = np.arange(h, dtype="<i4").view(np.uint8).reshape(h, 4)
    blocks[:, 4:8] = np.frombuffer(struct.pack("<i", row_bytes), np.uint8)
    blocks[:, 8:] = rows.astype("<f4").view(np.uint8).reshape(h, row_bytes)
    with open(path, "wb") as f:
        f.write(header)
        f.write(offsets.astype("<u8").tobytes())
        f.write(blocks.tobytes())


def load_exr(path: str) -> tuple[np.ndarray, list]:
    """Reads an uncompressed scanline EXR of float channels; returns the planes
    in file order (C, H, W) and the channel names."""
    data = open(path, "rb").read()
    magic, version = struct.unpack_from("<ii", data, 0)
    if magic != _MAGIC or (version & 0xff) != 2 or version & 0x200:
        raise ValueError("not a single-part scanline OpenEXR file")
    pos = 8
    attrs = {}
    while data[pos] != 0:
        end = data.index(b"\0", pos)
        name = data[pos:end].decode()
        tend = data.index(b"\0", end + 1)
        kind = data[end + 1:tend].decode()
        size, = struct.unpack_from("<i", data, tend + 1)
        attrs[name] = (kind, data[tend + 5:tend + 5 + size])
        pos = tend + 5 + size
    pos += 1
    names, p = [], attrs["channels"][1]
    q = 0
    while p[q] != 0:
        end = p.index(b"\0", q)
        names.append(p[q:end].decode())
        ptype, = struct.unpack_from("<i", p, end + 1)
        if ptype != _FLOAT:
            raise ValueError("only float channels are supported")
        q = end + 1 + 16
    if attrs["compression"][1] != b"\0":
        raise ValueError("only uncompressed files are supported")
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    w, h, c = x1 - x0 + 1, y1 - y0 + 1, len(names)
    offsets = np.frombuffer(data, "<u8", h, pos)
    out = np.empty((c, h, w), np.float32)
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, int(off))
        row = np.frombuffer(data, "<f4", c * w, int(off) + 8).reshape(c, w)
        out[:, y - y0, :] = row
    return out, names
