"""ctypes binding of the C ABI in ``include/imageproc_b200.h``.

The shared library is the product: it is loaded from the package directory
and nothing else is ever substituted for it. A missing library raises
``ImportError`` at first use; there is no CPU or PyTorch fallback.
"""

from __future__ import annotations

import ctypes as C
import weakref

import numpy as np
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libimageproc_b200.so"

# ipb_status codes
OK = 0
ERR_TEMPLATE_WIDTH = 1
ERR_TEMPLATE_HEIGHT = 2
ERR_MASK_SIZE = 3
ERR_EMPTY_IMAGE = 4
ERR_INVALID_ARGUMENT = 5
ERR_CUDA = 6
ERR_NO_DEVICE = 7
ERR_OUT_OF_MEMORY = 8
ERR_TIMEOUT = 9

PANIC_CODES = {ERR_TEMPLATE_WIDTH, ERR_TEMPLATE_HEIGHT, ERR_MASK_SIZE, ERR_EMPTY_IMAGE}

# element type suffix -> (ctypes scalar, numpy dtype name)
EXTREMES_TYPES = {
    "u8": (C.c_uint8, "uint8"),
    "u16": (C.c_uint16, "uint16"),
    "u32": (C.c_uint32, "uint32"),
    "u64": (C.c_uint64, "uint64"),
    "i8": (C.c_int8, "int8"),
    "i16": (C.c_int16, "int16"),
    "i32": (C.c_int32, "int32"),
    "i64": (C.c_int64, "int64"),
    "f32": (C.c_float, "float32"),
    "f64": (C.c_double, "float64"),
}


class Panic(AssertionError):
    """A failed argument check: the condition on which the reference panics.

    The message is the reference's own assertion message.
    """


class DeviceError(RuntimeError):
    """A CUDA failure, or no usable sm_100 device."""


def _extremes_struct(ctype):
    class Extremes(C.Structure):
        _fields_ = [
            ("max_value", ctype),
            ("min_value", ctype),
            ("max_value_location_x", C.c_uint32),
            ("max_value_location_y", C.c_uint32),
            ("min_value_location_x", C.c_uint32),
            ("min_value_location_y", C.c_uint32),
        ]

    return Extremes


EXTREMES_STRUCTS = {k: _extremes_struct(v[0]) for k, v in EXTREMES_TYPES.items()}


class KernelStats(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("launches", C.c_uint64),
        ("total_ms", C.c_double),
        ("algorithmic_macs", C.c_double),
        ("algorithmic_bytes", C.c_double),
    ]


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    return int(lib().ipb_launch_count())


def profile_enable(on: bool) -> None:
    check(lib().ipb_profile_enable(int(bool(on))))


def profile_collect() -> dict[str, dict]:
    """Per-kernel timed launches since the last collect (then reset)."""
    buf = (KernelStats * 32)()
    n = lib().ipb_profile_collect(buf, 32)
    return {buf[k].name.decode(): {"launches": buf[k].launches, "total_ms": buf[k].total_ms,
                                   "algorithmic_macs": buf[k].algorithmic_macs,
                                   "algorithmic_bytes": buf[k].algorithmic_bytes}
            for k in range(min(n, 32))}


class TensorPlan(C.Structure):
    _fields_ = [(name, C.c_uint32) for name in (
        "tile_rows", "image_rows", "rows_per_stage", "stages", "image_buffers", "tmem_columns",
        "smem_bytes")]


def tensor_plan(w: int, h: int, masked: bool, batch: bool) -> dict | None:
    """The tensor-core tile plan of a w x h template (ipb_tensor_plan_for):
    host arithmetic, no device work. None when the tensor path does not take
    the shape."""
    out = TensorPlan()
    st = lib().ipb_tensor_plan_for(w, h, int(bool(masked)), int(bool(batch)), C.byref(out))
    if st == ERR_INVALID_ARGUMENT:
        return None
    check(st)
    return {name: int(getattr(out, name)) for name, _ in TensorPlan._fields_}


def tensor_set_plan(w: int, h: int, masked: bool, problems_per_set: int) -> dict | None:
    """The tile plan of a batch group computing pairs on one image in sets of
    `problems_per_set` (ipb_tensor_set_plan_for): host arithmetic. None when
    no such plan fits."""
    out = TensorPlan()
    f = lib().ipb_tensor_set_plan_for
    f.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.c_uint32, C.c_void_p]
    st = f(w, h, int(bool(masked)), problems_per_set, C.byref(out))
    if st == ERR_INVALID_ARGUMENT:
        return None
    check(st)
    return {name: int(getattr(out, name)) for name, _ in TensorPlan._fields_}


_lib = None

u32 = C.c_uint32


def lib() -> C.CDLL:
    """Load (once) and return the shared library."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m imageproc_b200.build` "
            "(there is no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    L.ipb_last_error_message.restype = C.c_char_p
    L.ipb_version.restype = C.c_char_p
    L.ipb_set_precision.argtypes = [C.c_int]
    L.ipb_get_precision.restype = C.c_int
    L.ipb_set_path.argtypes = [C.c_int]
    L.ipb_get_path.restype = C.c_int
    L.ipb_launch_count.restype = C.c_uint64
    L.ipb_profile_enable.argtypes = [C.c_int]
    L.ipb_profile_collect.argtypes = [C.POINTER(KernelStats), C.c_int]
    L.ipb_profile_collect.restype = C.c_int
    # host buffers go in as plain addresses (numpy's .ctypes.data): building
    # a typed ctypes pointer per argument costs microseconds per call
    vp = C.c_void_p
    host = [vp, u32, u32, vp, u32, u32, C.c_int]
    for name in ("ipb_match_template", "ipb_match_template_parallel"):
        getattr(L, name).argtypes = host + [vp]
        getattr(L, name).restype = C.c_int
    for name in ("ipb_match_template_with_mask", "ipb_match_template_with_mask_parallel"):
        getattr(L, name).argtypes = host + [vp, u32, u32, vp]
        getattr(L, name).restype = C.c_int
    L.ipb_match_template_device.argtypes = [
        C.c_void_p, u32, u32, C.c_void_p, u32, u32, C.c_void_p, u32, u32, C.c_int, C.c_int,
        C.c_int, C.c_void_p, C.c_void_p]
    L.ipb_match_template_device.restype = C.c_int
    L.ipb_match_template_device_noalloc.argtypes = L.ipb_match_template_device.argtypes
    L.ipb_match_template_device_noalloc.restype = C.c_int
    for suf, (ct, _) in EXTREMES_TYPES.items():
        f = getattr(L, f"ipb_find_extremes_{suf}")
        f.argtypes = [C.c_void_p, u32, u32, C.POINTER(EXTREMES_STRUCTS[suf])]
        f.restype = C.c_int
        f = getattr(L, f"ipb_find_extremes_{suf}_device")
        f.argtypes = [C.c_void_p, u32, u32, C.POINTER(EXTREMES_STRUCTS[suf]), C.c_void_p]
        f.restype = C.c_int
    L.ipb_host_alloc.argtypes = [C.c_size_t]
    L.ipb_host_alloc.restype = C.c_void_p
    L.ipb_host_free.argtypes = [C.c_void_p]
    L.ipb_host_free.restype = None
    L.ipb_host_cache_release.argtypes = []
    L.ipb_host_cache_release.restype = None
    L.ipb_tensor_plan_for.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.POINTER(TensorPlan)]
    L.ipb_debug_set_pipeline_wait_ns.argtypes = [C.c_uint64]
    L.ipb_debug_set_pipeline_wait_ns.restype = None
    L.ipb_debug_stall_pipelines.argtypes = [C.c_int]
    L.ipb_debug_stall_pipelines.restype = None
    _lib = L
    return L


def host_empty(shape, dtype=np.float32) -> np.ndarray:
    """An uninitialised array in page-locked memory from the library's cache
    (ipb_host_alloc), returned to the cache when the last view of it is gone;
    ordinary memory when no CUDA device is usable. The device writes such
    buffers at the full link rate, with no first-touch page faults."""
    dt = np.dtype(dtype)
    n = int(np.prod(shape)) * dt.itemsize
    L = lib()
    p = L.ipb_host_alloc(n) if n else None
    if not p:
        return np.empty(shape, dt)
    raw = (C.c_char * n).from_address(p)
    weakref.finalize(raw, L.ipb_host_free, p)
    return np.frombuffer(raw, dtype=dt).reshape(shape)


def check(status: int) -> None:
    """Raise for a non-zero ipb_status, with the library's message."""
    if status == OK:
        return
    msg = lib().ipb_last_error_message().decode()
    if status in PANIC_CODES:
        raise Panic(msg)
    if status == ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    raise DeviceError(f"[ipb status {status}] {msg}")
