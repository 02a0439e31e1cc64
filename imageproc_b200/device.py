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


# ---- batches ------------------------------------------------------------------

class _Pair(C.Structure):
    _fields_ = [
        ("image", C.c_void_p), ("image_width", C.c_uint32), ("image_height", C.c_uint32),
        ("templ", C.c_void_p), ("template_width", C.c_uint32), ("template_height", C.c_uint32),
        ("mask", C.c_void_p), ("mask_width", C.c_uint32), ("mask_height", C.c_uint32),
        ("mask_is_binary", C.c_int), ("method", C.c_int),
        ("out", C.c_void_p), ("extremes", C.c_void_p),
    ]


EXTREMES_DTYPE = [("max_value", "<f4"), ("min_value", "<f4"), ("max_x", "<u4"), ("max_y", "<u4"),
                  ("min_x", "<u4"), ("min_y", "<u4")]


class _BatchGroup(C.Structure):
    _fields_ = [("row_width", C.c_uint32), ("tile_rows", C.c_uint32), ("masked", C.c_int),
                ("pairs", C.c_uint32), ("tiles", C.c_uint32), ("set_size", C.c_uint32)]


def _bind_batch():
    L = _lib.lib()
    if getattr(L, "_batch_bound", False):
        return L
    L.ipb_match_template_batch_device.argtypes = [C.POINTER(_Pair), C.c_uint32, C.c_int, C.c_void_p]
    L.ipb_match_template_batch_device.restype = C.c_int
    L.ipb_batch_plan_create.argtypes = [C.POINTER(_Pair), C.c_uint32, C.c_int, C.POINTER(C.c_void_p)]
    L.ipb_batch_plan_create.restype = C.c_int
    L.ipb_batch_plan_launch.argtypes = [C.c_void_p, C.c_void_p]
    L.ipb_batch_plan_launch.restype = C.c_int
    L.ipb_batch_plan_info.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.ipb_batch_plan_info.restype = C.c_int
    L.ipb_batch_plan_groups.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(_BatchGroup), C.POINTER(C.c_uint32)]
    L.ipb_batch_plan_groups.restype = C.c_int
    L.ipb_batch_plan_destroy.argtypes = [C.c_void_p]
    L.ipb_batch_plan_destroy.restype = C.c_int
    L._batch_bound = True
    return L


class Batch:
    """A batch of (image, template[, mask], method) pairs on the device.

    ``items``: sequence of ``(image, template, method)`` or
    ``(image, template, method, mask)`` CUDA uint8 tensors. Score maps are
    allocated here (``self.outs``) and, with ``extremes=True``, each map's
    find_extremes record is written on the device into ``self.extremes``
    (an int32 tensor of n x 6 words; see :meth:`extremes_host`).
    """

    def __init__(self, items, *, extremes: bool = True, masks_binary: bool = True):
        self.items = list(items)
        dev = self.items[0][0].device if self.items else torch.device("cuda")
        self.outs = []
        n = len(self.items)
        self.extremes = torch.zeros((max(n, 1), 6), dtype=torch.int32, device=dev)
        self._pairs = (_Pair * max(n, 1))()
        for i, it in enumerate(self.items):
            image, template, method = it[0], it[1], it[2]
            mask = it[3] if len(it) > 3 else None
            _check_gray(image, "image")
            _check_gray(template, "template")
            H, W = image.shape
            h, w = template.shape
            out = torch.empty((max(H - h + 1, 1), max(W - w + 1, 1)), dtype=torch.float32,
                              device=image.device)
            self.outs.append(out)
            p = self._pairs[i]
            p.image, p.image_width, p.image_height = image.data_ptr(), W, H
            p.templ, p.template_width, p.template_height = template.data_ptr(), w, h
            if mask is not None:
                _check_gray(mask, "mask")
                p.mask, p.mask_height, p.mask_width = mask.data_ptr(), mask.shape[0], mask.shape[1]
                p.mask_is_binary = int(masks_binary)
            p.method = int(MatchTemplateMethod(method))
            p.out = out.data_ptr()
            p.extremes = (self.extremes.data_ptr() + 24 * i) if extremes else None

    def run(self, precision: Precision | int = Precision.ExactFp64, stream=None):
        """One-shot batch (returns when the batch has completed)."""
        L = _bind_batch()
        check(L.ipb_match_template_batch_device(self._pairs, len(self.items), int(precision),
                                                _stream_handle(stream)))
        return self.outs

    def extremes_host(self):
        """The find_extremes records as a list of Extremes."""
        import numpy as np
        raw = self.extremes[: len(self.items)].cpu().numpy().view(np.dtype(EXTREMES_DTYPE)).reshape(-1)
        return [Extremes(float(r["max_value"]), float(r["min_value"]), (int(r["max_x"]), int(r["max_y"])),
                         (int(r["min_x"]), int(r["min_y"]))) for r in raw]


class BatchPlan:
    """A planned batch replayed as a CUDA graph (ipb_batch_plan_*)."""

    def __init__(self, batch: Batch, precision: Precision | int = Precision.ExactFp64):
        L = _bind_batch()
        self.batch = batch
        self._h = C.c_void_p()
        check(L.ipb_batch_plan_create(batch._pairs, len(batch.items), int(precision), C.byref(self._h)))

    def launch(self, stream=None):
        check(_bind_batch().ipb_batch_plan_launch(self._h, _stream_handle(stream)))
        return self.batch.outs

    def info(self):
        """Kernels per launch, tensor-core pairs and the tensor-core launches
        (row width, tile rows, mask kind, pairs, tiles) in launch order."""
        L = _bind_batch()
        k, t, n = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(L.ipb_batch_plan_info(self._h, C.byref(k), C.byref(t)))
        check(L.ipb_batch_plan_groups(self._h, 0, None, C.byref(n)))
        groups = (_BatchGroup * max(n.value, 1))()
        check(L.ipb_batch_plan_groups(self._h, n.value, groups, C.byref(n)))
        return {"kernels": k.value, "tensor_pairs": t.value,
                "launches": [{"row_width": g.row_width, "tile_rows": g.tile_rows, "masked": bool(g.masked),
                              "pairs": g.pairs, "tiles": g.tiles, "set_size": g.set_size}
                             for g in groups[: n.value]]}

    def close(self):
        if self._h:
            _bind_batch().ipb_batch_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def match_templates_device(image: torch.Tensor, templates: torch.Tensor, method, *,
                           precision: Precision | int = Precision.ExactFp64, scores: bool = True,
                           extremes: bool = False, out: torch.Tensor | None = None, stream=None):
    """Score n templates of one size (an (n, h, w) uint8 CUDA tensor) against
    one image in one tensor-core launch (ipb_match_templates_device).

    Returns ``(scores, extremes)``: scores is position-major, shape
    (H - h + 1, W - w + 1, n) (None when ``scores=False``); extremes is a list
    of n :class:`Extremes` (None unless ``extremes=True``)."""
    L = _lib.lib()
    if not getattr(L, "_many_bound", False):
        L.ipb_match_templates_device.argtypes = [
            C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
            C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ipb_match_templates_device.restype = C.c_int
        L._many_bound = True
    _check_gray(image, "image")
    if templates.dtype != torch.uint8 or templates.dim() != 3 or not templates.is_cuda or \
            not templates.is_contiguous():
        raise TypeError("templates must be a contiguous (n, h, w) uint8 CUDA tensor")
    H, W = image.shape
    n, h, w = templates.shape
    if scores and out is None:
        out = torch.empty((max(H - h + 1, 1), max(W - w + 1, 1), n), dtype=torch.float32,
                          device=image.device)
    ext = torch.zeros((n, 6), dtype=torch.int32, device=image.device) if extremes else None
    check(L.ipb_match_templates_device(
        image.data_ptr(), W, H, templates.data_ptr(), w, h, n, int(MatchTemplateMethod(method)),
        int(precision), out.data_ptr() if scores else None, ext.data_ptr() if extremes else None,
        _stream_handle(stream)))
    ex = None
    if extremes:
        import numpy as np
        raw = ext.cpu().numpy().view(np.dtype(EXTREMES_DTYPE)).reshape(-1)
        ex = [Extremes(float(r["max_value"]), float(r["min_value"]), (int(r["max_x"]), int(r["max_y"])),
                       (int(r["min_x"]), int(r["min_y"]))) for r in raw]
    return (out if scores else None), ex
