"""imageproc's ``integral_image`` module on the GPU (src/integral_image.rs).

``integral_image`` / ``integral_squared_image`` (:50, :89) build the table on
the device (ipb_integral_image_u32 / _u64); ``sum_image_pixels`` (:250) and
``variance`` (:303) are the reference's O(1) lookups into such a table.

Images are (H, W) arrays (Luma) or (H, W, C) arrays with C = 3 (Rgb) or 4
(Rgba) of uint8. Tables are (H+1, W+1) or (H+1, W+1, C) of uint32 (wrapping
modulo 2^32 like the reference's u32 sums in a release build) or uint64.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

_FNS = {(np.dtype(np.uint32), False): "ipb_integral_image_u32",
        (np.dtype(np.uint32), True): "ipb_integral_squared_image_u32",
        (np.dtype(np.uint64), False): "ipb_integral_image_u64",
        (np.dtype(np.uint64), True): "ipb_integral_squared_image_u64"}


def _table(image, square: bool, dtype) -> np.ndarray:
    a = np.ascontiguousarray(image)
    if a.dtype != np.uint8 or a.ndim not in (2, 3) or (a.ndim == 3 and a.shape[2] not in (3, 4)):
        raise TypeError("integral images take (H, W) or (H, W, 3|4) uint8 images")
    dt = np.dtype(dtype)
    if dt not in (np.dtype(np.uint32), np.dtype(np.uint64)):
        raise TypeError("integral images are uint32 or uint64")
    H, W = a.shape[:2]
    ch = 1 if a.ndim == 2 else a.shape[2]
    L = _lib.lib()
    fn = getattr(L, _FNS[(dt, square)])
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]
    fn.restype = C.c_int
    shape = (H + 1, W + 1) if ch == 1 else (H + 1, W + 1, ch)
    out = _lib.host_empty(shape, dt)
    check(fn(a.ctypes.data if a.size else None, W, H, ch, out.ctypes.data))
    return out


def integral_image(image, dtype=np.uint32) -> np.ndarray:
    """``integral_image`` (src/integral_image.rs:50): entry (x, y) holds the sum
    of the pixels strictly above and to the left of (x, y)."""
    return _table(image, False, dtype)


def integral_squared_image(image, dtype=np.uint32) -> np.ndarray:
    """``integral_squared_image`` (src/integral_image.rs:89): the same for the
    squares of the pixels."""
    return _table(image, True, dtype)


def sum_image_pixels(integral, left: int, top: int, right: int, bottom: int) -> np.ndarray:
    """``sum_image_pixels`` (src/integral_image.rs:250-271): per-channel sum
    over [left, right] x [top, bottom], I(r+1, b+1) + I(l, t) - I(r+1, t) -
    I(l, b+1) in the table's element arithmetic."""
    t = np.asarray(integral)
    px = (lambda x, y: np.atleast_1d(t[y, x]).copy())
    a, b = px(right + 1, bottom + 1), px(left, top)
    c, d = px(right + 1, top), px(left, bottom + 1)
    with np.errstate(over="ignore"):
        return (a + b) - c - d


def variance(integral, integral_squared, left: int, top: int, right: int, bottom: int) -> float:
    """``variance`` (src/integral_image.rs:303-315) of [left, right] x [top,
    bottom] from u32 Luma tables, in f64."""
    n = float(right - left + 1) * float(bottom - top + 1)
    sum_sq = float(sum_image_pixels(integral_squared, left, top, right, bottom)[0])
    s = float(sum_image_pixels(integral, left, top, right, bottom)[0])
    return (sum_sq - (s * s) / n) / n
