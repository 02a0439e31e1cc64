"""Device-resident entry points on torch CUDA tensors.

These wrap the ``_device`` functions of the C ABI: inputs and outputs stay in
HBM, work is enqueued on the caller's stream (torch's current stream by
default) and nothing is synchronised except ``find_extremes_device``, which
returns its record to the host. PyTorch only provides the device memory and
the stream; every kernel is the library's.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check
from .template_matching import Extremes, MatchTemplateMethod, Precision

_TORCH_SUFFIX = {
    torch.uint8: "u8", torch.uint16: "u16", torch.uint32: "u32", torch.uint64: "u64",
    torch.int8: "i8", torch.int16: "i16", torch.int32: "i32", torch.int64: "i64",
    torch.float32: "f32", torch.float64: "f64",
}


def _stream_handle(stream) -> int | None:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


def _check_gray(t: torch.Tensor, what: str) -> None:
    if t.dtype != torch.uint8 or t.dim() != 2 or not t.is_cuda or not t.is_contiguous():
        raise TypeError(f"{what} must be a contiguous 2-D uint8 CUDA tensor")


def match_template_device(image: torch.Tensor, template: torch.Tensor, method,
                          mask: torch.Tensor | None = None, *, mask_is_binary: bool = False,
                          precision: Precision | int = Precision.ExactFp64,
                          out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Score map of ``template`` over ``image`` (match_template /
    match_template_with_mask, src/template_matching.rs:78, :125)."""
    _check_gray(image, "image")
    _check_gray(template, "template")
    H, W = image.shape
    h, w = template.shape
    mh = mw = 0
    if mask is not None:
        _check_gray(mask, "mask")
        mh, mw = mask.shape
    if out is None:
        shape = (max(H - h + 1, 1), max(W - w + 1, 1))
        out = torch.empty(shape, dtype=torch.float32, device=image.device)
    check(_lib.lib().ipb_match_template_device(
        image.data_ptr(), W, H, template.data_ptr(), w, h,
        mask.data_ptr() if mask is not None else None, mw, mh, int(bool(mask_is_binary)),
        int(MatchTemplateMethod(method)), int(precision), out.data_ptr(), _stream_handle(stream)))
    return out


def find_extremes_device(image: torch.Tensor, stream=None) -> Extremes:
    """find_extremes (src/template_matching.rs:479-511) of a 2-D CUDA tensor."""
    if image.dim() != 2 or not image.is_cuda or not image.is_contiguous():
        raise TypeError("find_extremes_device takes a contiguous 2-D CUDA tensor")
    suf = _TORCH_SUFFIX[image.dtype]
    H, W = image.shape
    res = _lib.EXTREMES_STRUCTS[suf]()
    fn = getattr(_lib.lib(), f"ipb_find_extremes_{suf}_device")
    check(fn(image.data_ptr() if image.numel() else None, W, H, C.byref(res),
             _stream_handle(stream)))
    return Extremes(res.max_value, res.min_value,
                    (res.max_value_location_x, res.max_value_location_y),
                    (res.min_value_location_x, res.min_value_location_y))
