"""imageproc's ``filter_clamped`` family on the GPU (src/filter/mod.rs).

``filter_clamped`` (:202) correlates a u8 image -- (H, W) Luma or (H, W, 3|4)
Rgb/Rgba -- with a 2-D kernel (float32 or int32 array, row-major, any size),
padding by continuity, accumulating in the kernel's type in the reference's
order and clamping to ``out_dtype`` with the reference's ``Clamp``. The 1-D
forms follow from it exactly: ``horizontal_filter`` (:232) is a 1 x n kernel,
``vertical_filter`` (:319) an n x 1 kernel, both clamped to u8 like the
source, and ``separable_filter`` (:169) is the vertical filter of the
horizontal one, as in the reference. ``laplacian_filter`` (:440) is the 3 x 3
Laplacian into i16.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Panic, check

_ELEM = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.int16): 5, np.dtype(np.int32): 6,
         np.dtype(np.float32): 8}
_KTYPE = {np.dtype(np.float32): 0, np.dtype(np.int32): 1}


def filter_clamped(image, kernel, out_dtype=np.uint8) -> np.ndarray:
    """``filter_clamped`` (src/filter/mod.rs:202-212)."""
    a = np.ascontiguousarray(image)
    if a.dtype != np.uint8 or a.ndim not in (2, 3) or (a.ndim == 3 and a.shape[2] not in (3, 4)):
        raise TypeError("filter_clamped takes (H, W) or (H, W, 3|4) uint8 images")
    k = np.ascontiguousarray(kernel)
    if k.ndim != 2 or k.dtype not in _KTYPE:
        raise TypeError("kernels are 2-D float32 or int32 arrays")
    od = np.dtype(out_dtype)
    if od not in _ELEM:
        raise TypeError(f"unsupported output type {od}")
    H, W = a.shape[:2]
    ch = 1 if a.ndim == 2 else a.shape[2]
    kh, kw = k.shape
    if kh == 0 or kw == 0:  # Kernel::new (src/kernel.rs:24-33)
        raise Panic("width and height must be non-zero")
    out = _lib.host_empty(a.shape, od)
    L = _lib.lib()
    L.ipb_filter_clamped.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_int,
                                     C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
    L.ipb_filter_clamped.restype = C.c_int
    check(L.ipb_filter_clamped(a.ctypes.data if a.size else None, W, H, ch, k.ctypes.data if k.size else None,
                               _KTYPE[k.dtype], kw, kh, _ELEM[od], out.ctypes.data if out.size else None))
    return out


def horizontal_filter(image, kernel) -> np.ndarray:
    """``horizontal_filter`` (src/filter/mod.rs:232-316): a 1 x n kernel, u8 out."""
    k = np.ascontiguousarray(kernel)
    return filter_clamped(image, k.reshape(1, -1), np.uint8)


def vertical_filter(image, kernel) -> np.ndarray:
    """``vertical_filter`` (src/filter/mod.rs:319-404): an n x 1 kernel, u8 out."""
    k = np.ascontiguousarray(kernel)
    return filter_clamped(image, k.reshape(-1, 1), np.uint8)


def separable_filter(image, h_kernel, v_kernel) -> np.ndarray:
    """``separable_filter`` (src/filter/mod.rs:169-181): horizontal, then vertical."""
    if np.size(h_kernel) != np.size(v_kernel):
        raise Panic("the two 1D kernels must be the same length")
    return vertical_filter(horizontal_filter(image, h_kernel), v_kernel)


def separable_filter_equal(image, kernel) -> np.ndarray:
    """``separable_filter_equal`` (src/filter/mod.rs:188-195)."""
    return separable_filter(image, kernel, kernel)


LAPLACIAN = np.array([[0, 1, 0], [1, -4, 1], [0, 1, 0]], np.int32)


def laplacian_filter(image) -> np.ndarray:
    """``laplacian_filter`` (src/filter/mod.rs:440-445): i16 out."""
    return filter_clamped(image, LAPLACIAN, np.int16)
