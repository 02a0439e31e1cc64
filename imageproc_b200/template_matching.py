"""imageproc's ``template_matching`` module, backed by sm_100a kernels.

Mirrors imageproc 0.27.0 ``src/template_matching.rs``: same names, same
argument meaning, same panics (raised here as :class:`Panic` with the
reference's assertion message), same output size
``(image.width - template.width + 1) x (image.height - template.height + 1)``.

A ``GrayImage`` is a C-contiguous ``numpy.uint8`` array of shape
``(height, width)``; an ``Image<Luma<f32>>`` is a ``numpy.float32`` array of
the same orientation. Locations are ``(x, y)`` like the reference's.

Every call goes through the C ABI to the CUDA library; results are
identical for the serial and ``_parallel`` forms, as in the reference.
"""

from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import _lib
from ._lib import Panic, check

__all__ = [
    "MatchTemplateMethod", "Extremes", "Panic", "Precision",
    "match_template", "match_template_parallel",
    "match_template_with_mask", "match_template_with_mask_parallel",
    "find_extremes", "set_precision", "get_precision", "Path", "set_path", "get_path",
]


class MatchTemplateMethod(enum.IntEnum):
    """Scoring functions (src/template_matching.rs:8-64), same order."""

    SumOfSquaredErrors = 0
    SumOfSquaredErrorsNormalized = 1
    CrossCorrelation = 2
    CrossCorrelationNormalized = 3


class Precision(enum.IntEnum):
    """Arithmetic of the score maps (see include/imageproc_b200.h)."""

    ExactFp64 = 0
    ExactF32 = 1
    ReferenceF32 = 2


@dataclass(frozen=True)
class Extremes:
    """``Extremes<T>`` (src/template_matching.rs:463-475)."""

    max_value: Any
    min_value: Any
    max_value_location: tuple[int, int]
    min_value_location: tuple[int, int]


def set_precision(precision: Precision | int) -> None:
    """Process-wide precision of the reference-shaped functions."""
    check(_lib.lib().ipb_set_precision(int(precision)))


def get_precision() -> Precision:
    return Precision(_lib.lib().ipb_get_precision())


class Path(enum.IntEnum):
    """Kernel family of the exact precisions (identical results)."""

    Auto = 0
    CudaCores = 1
    TensorCores = 2
    RowOperand = 3


def set_path(path: Path | int) -> None:
    check(_lib.lib().ipb_set_path(int(path)))


def get_path() -> Path:
    return Path(_lib.lib().ipb_get_path())


def _gray(img: np.ndarray, what: str) -> np.ndarray:
    a = np.asarray(img)
    if a.dtype != np.uint8 or a.ndim != 2:
        raise TypeError(f"{what} must be a 2-D uint8 array (GrayImage), got {a.dtype} {a.shape}")
    return np.ascontiguousarray(a)


def _ptr(a: np.ndarray):
    return a.ctypes.data  # numpy gives empty arrays an address too


def _run(fn_name: str, image, template, method, mask=None) -> np.ndarray:
    image = _gray(image, "image")
    template = _gray(template, "template")
    H, W = image.shape
    h, w = template.shape
    m = MatchTemplateMethod(method)
    L = _lib.lib()
    fn = getattr(L, fn_name)
    # the reference asserts before allocating its output; so does the library,
    # so size the output only for valid shapes
    if mask is not None:
        mask = _gray(mask, "mask")
        mh, mw = mask.shape
        valid = (mh, mw) == (h, w) and W >= w and H >= h
        out = _lib.host_empty((H - h + 1, W - w + 1) if valid else (1, 1))
        check(fn(_ptr(image), W, H, _ptr(template), w, h, int(m), _ptr(mask), mw, mh, _ptr(out)))
        return out
    valid = W >= w and H >= h
    out = _lib.host_empty((H - h + 1, W - w + 1) if valid else (1, 1))
    check(fn(_ptr(image), W, H, _ptr(template), w, h, int(m), _ptr(out)))
    return out


def match_template(image, template, method) -> np.ndarray:
    """``match_template`` (src/template_matching.rs:78-92)."""
    return _run("ipb_match_template", image, template, method)


def match_template_parallel(image, template, method) -> np.ndarray:
    """``match_template_parallel`` (src/template_matching.rs:96-110)."""
    return _run("ipb_match_template_parallel", image, template, method)


def match_template_with_mask(image, template, method, mask) -> np.ndarray:
    """``match_template_with_mask`` (src/template_matching.rs:125-140)."""
    return _run("ipb_match_template_with_mask", image, template, method, mask)


def match_template_with_mask_parallel(image, template, method, mask) -> np.ndarray:
    """``match_template_with_mask_parallel`` (src/template_matching.rs:144-163)."""
    return _run("ipb_match_template_with_mask_parallel", image, template, method, mask)


_DTYPE_SUFFIX = {np.dtype(v[1]): k for k, v in _lib.EXTREMES_TYPES.items()}


def find_extremes(image: np.ndarray) -> Extremes:
    """``find_extremes`` (src/template_matching.rs:479-511) for any Primitive
    channel type (numpy uint8..uint64, int8..int64, float32, float64)."""
    a = np.ascontiguousarray(np.asarray(image))
    if a.ndim != 2:
        raise TypeError("find_extremes takes a single-channel 2-D image")
    suf = _DTYPE_SUFFIX.get(a.dtype)
    if suf is None:
        raise TypeError(f"unsupported channel type {a.dtype}")
    H, W = a.shape
    res = _lib.EXTREMES_STRUCTS[suf]()
    fn = getattr(_lib.lib(), f"ipb_find_extremes_{suf}")
    check(fn(a.ctypes.data_as(C.c_void_p) if a.size else None, W, H, C.byref(res)))
    cast = a.dtype.type
    return Extremes(cast(res.max_value), cast(res.min_value),
                    (res.max_value_location_x, res.max_value_location_y),
                    (res.min_value_location_x, res.min_value_location_y))
