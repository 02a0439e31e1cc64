"""imageproc's ``suppress`` module on the GPU (src/suppress.rs).

``suppress_non_maximum`` (:10) takes an (H, W) array of any integer channel
type (and, additively, float32 score maps, compared in IEEE total order:
-0 below +0, NaN above every number) and returns an array of the same
type that keeps a pixel's value where it is the greatest in the
(2 * radius + 1)^2 window centred on it and is zero elsewhere; among equal
values the lexicographically smaller (x, y) wins.

``local_maxima`` (:111) takes scored points -- objects with ``x``, ``y`` and
``score`` attributes, or (x, y, score) tuples -- and returns the points that
have the highest score in the window centred on them, in the reference's
order (sorted by (y, x)).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

_SUFFIX = {np.dtype(t): s for t, s in (
    (np.uint8, "u8"), (np.uint16, "u16"), (np.uint32, "u32"), (np.uint64, "u64"),
    (np.int8, "i8"), (np.int16, "i16"), (np.int32, "i32"), (np.int64, "i64"), (np.float32, "f32"))}


def suppress_non_maximum(image, radius: int) -> np.ndarray:
    """``suppress_non_maximum`` (src/suppress.rs:10-77)."""
    a = np.ascontiguousarray(image)
    if a.ndim != 2 or a.dtype not in _SUFFIX:
        raise TypeError(f"suppress_non_maximum takes a 2-D array of {sorted(str(d) for d in _SUFFIX)}")
    H, W = a.shape
    out = _lib.host_empty((H, W), a.dtype)
    if a.size == 0:
        return out
    fn = getattr(_lib.lib(), f"ipb_suppress_non_maximum_{_SUFFIX[a.dtype]}")
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]
    fn.restype = C.c_int
    check(fn(a.ctypes.data, W, H, int(radius), out.ctypes.data))
    return out


def _coords(points):
    xs, ys, sc = [], [], []
    for p in points:
        if hasattr(p, "x"):
            x, y, s = p.x, p.y, p.score
        else:
            x, y, s = p
        xs.append(x)
        ys.append(y)
        sc.append(s)
    return (np.asarray(xs, np.uint32), np.asarray(ys, np.uint32), np.asarray(sc, np.float32))


def local_maxima_indices(xs, ys, scores, radius: int) -> list[int]:
    """Indices (into the inputs) of the points local_maxima keeps, in its order."""
    xs = np.ascontiguousarray(xs, np.uint32)
    ys = np.ascontiguousarray(ys, np.uint32)
    sc = np.ascontiguousarray(scores, np.float32)
    n = len(xs)
    if not (len(ys) == n == len(sc)):
        raise ValueError("xs, ys and scores must have one entry per point")
    L = _lib.lib()
    L.ipb_local_maxima.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                   C.POINTER(C.c_uint32)]
    L.ipb_local_maxima.restype = C.c_int
    out = np.empty(max(n, 1), np.uint32)
    count = C.c_uint32(0)
    check(L.ipb_local_maxima(xs.ctypes.data if n else None, ys.ctypes.data if n else None,
                             sc.ctypes.data if n else None, n, int(radius), out.ctypes.data, C.byref(count)))
    return [int(i) for i in out[:count.value]]


def local_maxima(points, radius: int) -> list:
    """``local_maxima`` (src/suppress.rs:111-173)."""
    points = list(points)
    xs, ys, sc = _coords(points)
    return [points[i] for i in local_maxima_indices(xs, ys, sc, radius)]
