"""Host-side image files for the example workflow: 8-bit PNG (grayscale,
gray+alpha, RGB, RGBA; non-interlaced; every row filter) and 8-bit binary
netpbm (P5, P6), decoded to numpy arrays and encoded from them.

`to_luma8` converts to one 8-bit channel the way the `image` crate (0.25,
which the reference's example uses through `open(..).to_luma8()`) does:
alpha is dropped and RGB becomes (2126 R + 7152 G + 722 B) / 10000 in integer
arithmetic. That crate is not vendored with the reference; the formula is
restated from its published source.
"""

from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np

_SIG = b"\x89PNG\r\n\x1a\n"
_CHANNELS = {0: 1, 2: 3, 4: 2, 6: 4}


class ImageFormatError(ValueError):
    pass


def _unfilter(raw: bytes, width: int, height: int, bpp: int) -> np.ndarray:
    stride = width * bpp
    out = np.zeros((height, stride), np.uint8)
    prior = np.zeros(stride, np.int32)
    pos = 0
    for y in range(height):
        ftype = raw[pos]
        line = np.frombuffer(raw, np.uint8, stride, pos + 1).astype(np.int32)
        pos += 1 + stride
        if ftype == 0:
            cur = line
        elif ftype == 1:  # Sub: a running sum per channel
            cur = np.cumsum(line.reshape(width, bpp), axis=0).reshape(-1) & 0xFF
        elif ftype == 2:  # Up
            cur = (line + prior) & 0xFF
        elif ftype in (3, 4):  # Average, Paeth: each byte needs the one decoded before it
            cur = line.tolist()
            up = prior.tolist()
            for i in range(stride):
                a = cur[i - bpp] if i >= bpp else 0
                b = up[i]
                if ftype == 3:
                    pred = (a + b) >> 1
                else:
                    c = up[i - bpp] if i >= bpp else 0
                    p = a + b - c
                    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                    pred = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                cur[i] = (cur[i] + pred) & 0xFF
            cur = np.array(cur, np.int32)
        else:
            raise ImageFormatError(f"unknown PNG filter type {ftype}")
        out[y] = cur
        prior = cur.astype(np.int32)
    return out


def decode_png(data: bytes) -> np.ndarray:
    """(H, W) for grayscale, (H, W, C) otherwise."""
    if data[:8] != _SIG:
        raise ImageFormatError("not a PNG file")
    pos, idat, hdr = 8, [], None
    while pos < len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat.append(body)
        elif kind == b"IEND":
            break
    if hdr is None:
        raise ImageFormatError("PNG without IHDR")
    width, height, depth, ctype, _comp, _filt, interlace = hdr
    if depth != 8 or ctype not in _CHANNELS or interlace:
        raise ImageFormatError(f"unsupported PNG: bit depth {depth}, color type {ctype}, interlace {interlace}")
    ch = _CHANNELS[ctype]
    px = _unfilter(zlib.decompress(b"".join(idat)), width, height, ch)
    return px.reshape(height, width) if ch == 1 else px.reshape(height, width, ch)


def encode_png(img: np.ndarray) -> bytes:
    """8-bit grayscale (H, W) or RGB (H, W, 3), filter 0 on every row."""
    a = np.ascontiguousarray(img, np.uint8)
    if a.ndim == 2:
        ctype, ch = 0, 1
    elif a.ndim == 3 and a.shape[2] == 3:
        ctype, ch = 2, 3
    else:
        raise ImageFormatError("encode_png takes (H, W) or (H, W, 3) uint8 arrays")
    h, w = a.shape[:2]
    rows = np.zeros((h, 1 + w * ch), np.uint8)
    rows[:, 1:] = a.reshape(h, w * ch)

    def chunk(kind: bytes, body: bytes) -> bytes:
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    return (_SIG + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0))
            + chunk(b"IDAT", zlib.compress(rows.tobytes(), 6)) + chunk(b"IEND", b""))


def _decode_pnm(data: bytes) -> np.ndarray:
    fields, pos = [], 2
    while len(fields) < 3:
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            pos = data.index(b"\n", pos) + 1
            continue
        end = pos
        while not data[end:end + 1].isspace():
            end += 1
        fields.append(int(data[pos:end]))
        pos = end
    pos += 1  # the single whitespace byte before the raster
    w, h, maxval = fields
    if maxval != 255:
        raise ImageFormatError("only 8-bit netpbm files are supported")
    ch = 1 if data[:2] == b"P5" else 3
    px = np.frombuffer(data, np.uint8, w * h * ch, pos)
    return px.reshape(h, w) if ch == 1 else px.reshape(h, w, 3)


def read_image(path: str | Path) -> np.ndarray:
    data = Path(path).read_bytes()
    if data[:8] == _SIG:
        return decode_png(data)
    if data[:2] in (b"P5", b"P6"):
        return _decode_pnm(data)
    raise ImageFormatError(f"unsupported image file {path}")


def write_png(path: str | Path, img: np.ndarray) -> None:
    Path(path).write_bytes(encode_png(img))


def to_luma8(img: np.ndarray) -> np.ndarray:
    a = np.asarray(img, np.uint8)
    if a.ndim == 2:
        return a.copy()
    if a.shape[2] in (1, 2):  # Luma, LumaA: drop alpha
        return a[:, :, 0].copy()
    rgb = a[:, :, :3].astype(np.uint32)
    return ((2126 * rgb[:, :, 0] + 7152 * rgb[:, :, 1] + 722 * rgb[:, :, 2]) // 10000).astype(np.uint8)
