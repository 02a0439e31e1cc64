"""ctypes binding of the CPU oracle (``oracle/tm_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Imported by the
test-suite, the smoke check and the benchmark's CPU-baseline leg, never by
the ``imageproc_b200`` package.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libtm_oracle.so"

TYPE_CODES = {np.dtype(t): k for k, t in enumerate(
    ["uint8", "uint16", "uint32", "uint64", "int8", "int16", "int32", "int64", "float32", "float64"])}

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        u8p, f32p, u64p = C.c_void_p, C.c_void_p, C.c_void_p
        u32 = C.c_uint32
        L.tmo_match_reference.argtypes = [u8p, u32, u32, u8p, u32, u32, u8p, u32, u32, C.c_int,
                                          f32p, u32, u32, C.c_int]
        L.tmo_sums.argtypes = [u8p, u32, u32, u8p, u32, u32, u8p, u64p, u64p, u64p, C.c_int]
        L.tmo_match_exact.argtypes = [u8p, u32, u32, u8p, u32, u32, u8p, u32, u32, C.c_int, C.c_int,
                                      f32p, C.c_int]
        L.tmo_match_exact_fast.argtypes = [u8p, u32, u32, u8p, u32, u32, C.c_int, C.c_int,
                                           C.c_void_p, C.c_void_p, C.c_int]
        L.tmo_many_exact_fast.argtypes = [u8p, u32, u32, u8p, u32, u32, u32, C.c_int, C.c_int,
                                          u32, u32, C.c_void_p, C.c_void_p, C.c_int]
        L.tmo_finish.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64]
        L.tmo_finish.restype = C.c_float
        L.tmo_find_extremes_index.argtypes = [C.c_void_p, u32, u32, C.c_int,
                                              C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.nxo_integral_u32.argtypes = [u8p, u32, u32, u32, C.c_int, C.c_void_p]
        L.nxo_integral_u64.argtypes = [u8p, u32, u32, u32, C.c_int, C.c_void_p]
        L.nxo_suppress_non_maximum.argtypes = [C.c_void_p, u32, u32, u32, C.c_void_p]
        L.nxo_suppress_non_maximum_naive.argtypes = [C.c_void_p, u32, u32, u32, C.c_void_p]
        L.nxo_local_maxima.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, u32, u32, C.c_void_p]
        L.nxo_local_maxima.restype = u32
        L.nxo_filter_clamped.argtypes = [u8p, u32, u32, u32, C.c_void_p, C.c_int, u32, u32, C.c_int, C.c_void_p]
        _lib = L
    return _lib


def default_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


class OracleError(AssertionError):
    pass


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _dims(image, template, mask):
    image = np.ascontiguousarray(image, np.uint8)
    template = np.ascontiguousarray(template, np.uint8)
    if mask is not None:
        mask = np.ascontiguousarray(mask, np.uint8)
    return image, template, mask


def match_reference(image, template, method, mask=None, rows=None, threads=None) -> np.ndarray:
    """The reference's f32 scores (bit-exact restatement). ``rows`` = (begin,
    end) restricts the output rows (a bounded sample)."""
    image, template, mask = _dims(image, template, mask)
    H, W = image.shape
    h, w = template.shape
    mh, mw = mask.shape if mask is not None else (0, 0)
    Ho, Wo = H - h + 1, W - w + 1
    r0, r1 = rows if rows is not None else (0, Ho)
    out = np.empty((max(r1 - r0, 0), Wo), np.float32)
    st = lib().tmo_match_reference(_p(image), W, H, _p(template), w, h, _p(mask), mw, mh,
                                   int(method), _p(out), r0, r1,
                                   threads if threads is not None else default_threads())
    if st:
        raise OracleError(f"oracle status {st}")
    return out


def sums(image, template, mask=None, threads=None):
    """Exact (X, Y, TSS) integer sums."""
    image, template, mask = _dims(image, template, mask)
    H, W = image.shape
    h, w = template.shape
    X = np.empty((H - h + 1, W - w + 1), np.uint64)
    Y = np.empty_like(X)
    tss = C.c_uint64()
    st = lib().tmo_sums(_p(image), W, H, _p(template), w, h, _p(mask), _p(X), _p(Y),
                        C.byref(tss), threads if threads is not None else default_threads())
    if st:
        raise OracleError(f"oracle status {st}")
    return X, Y, tss.value


def match_exact(image, template, method, mask=None, precision=0, threads=None) -> np.ndarray:
    """Exact integer sums + FP64 (precision 0) or f32 (1) normalisation."""
    image, template, mask = _dims(image, template, mask)
    H, W = image.shape
    h, w = template.shape
    mh, mw = mask.shape if mask is not None else (0, 0)
    out = np.empty((H - h + 1, W - w + 1), np.float32)
    st = lib().tmo_match_exact(_p(image), W, H, _p(template), w, h, _p(mask), mw, mh,
                               int(method), int(precision), _p(out),
                               threads if threads is not None else default_threads())
    if st:
        raise OracleError(f"oracle status {st}")
    return out


class _Extremes(C.Structure):
    _fields_ = [("max_value", C.c_double), ("min_value", C.c_double),
                ("max_x", C.c_uint32), ("max_y", C.c_uint32),
                ("min_x", C.c_uint32), ("min_y", C.c_uint32)]


def match_exact_fast(image, template, method, precision=0, want_map=True, threads=None):
    """Unmasked exact scores through the fast oracle form (templates of at most
    66051 pixels): returns (map or None, extremes) where extremes is
    find_extremes of the f32 map, (max_value, min_value, (max_x, max_y),
    (min_x, min_y)). The scores equal match_exact's."""
    image = np.ascontiguousarray(image, dtype=np.uint8)
    template = np.ascontiguousarray(template, dtype=np.uint8)
    H, W = image.shape
    h, w = template.shape
    out = np.empty((H - h + 1, W - w + 1), np.float32) if want_map else None
    ext = _Extremes()
    st = lib().tmo_match_exact_fast(_p(image), W, H, _p(template), w, h, int(method),
                                    int(precision), _p(out), C.byref(ext),
                                    threads if threads is not None else default_threads())
    if st:
        raise OracleError(f"oracle status {st}")
    e = (np.float32(ext.max_value), np.float32(ext.min_value), (ext.max_x, ext.max_y),
         (ext.min_x, ext.min_y))
    return out, e


def many_exact_fast(image, templates, method, precision=0, rows=None, want_maps=False,
                    threads=None):
    """n unmasked templates of one size (an (n, h, w) u8 array) against one
    image through the fast oracle form, output rows [r0, r1) (default all).
    Returns (maps or None, extremes): maps (n, r1 - r0, Wo) f32, extremes a
    list of n find_extremes tuples over those rows, in full-map coordinates."""
    image = np.ascontiguousarray(image, dtype=np.uint8)
    templates = np.ascontiguousarray(templates, dtype=np.uint8)
    H, W = image.shape
    n, h, w = templates.shape
    r0, r1 = rows if rows is not None else (0, H - h + 1)
    maps = np.empty((n, r1 - r0, W - w + 1), np.float32) if want_maps else None
    ext = (_Extremes * n)()
    st = lib().tmo_many_exact_fast(_p(image), W, H, _p(templates), w, h, n, int(method),
                                   int(precision), r0, r1, _p(maps), ext,
                                   threads if threads is not None else default_threads())
    if st:
        raise OracleError(f"oracle status {st}")
    return maps, [(np.float32(e.max_value), np.float32(e.min_value), (e.max_x, e.max_y),
                   (e.min_x, e.min_y)) for e in ext]


def find_extremes(image):
    """(max_value, min_value, (max_x, max_y), (min_x, min_y))."""
    a = np.ascontiguousarray(image)
    H, W = a.shape
    imax, imin = C.c_uint64(), C.c_uint64()
    st = lib().tmo_find_extremes_index(_p(a), W, H, TYPE_CODES[a.dtype], C.byref(imax),
                                       C.byref(imin))
    if st:
        raise OracleError(f"oracle status {st}")
    flat = a.reshape(-1)
    return (flat[imax.value], flat[imin.value], (imax.value % W, imax.value // W),
            (imin.value % W, imin.value // W))


# ---- integral images and non-maximum suppression (next_oracle.c) ------------

def order_keys(a) -> np.ndarray:
    """u64 keys that compare like the values of `a` (any integer or float dtype)."""
    a = np.ascontiguousarray(a)
    if a.dtype.kind == "u":
        return a.astype(np.uint64)
    if a.dtype.kind == "i":
        return a.astype(np.int64).view(np.uint64) ^ np.uint64(1 << 63)
    if a.dtype == np.float32:
        b = a.view(np.uint32).astype(np.uint64)
        return np.where(b >> np.uint64(31), ~b & np.uint64(0xFFFFFFFF), b | np.uint64(0x80000000))
    if a.dtype == np.float64:
        b = a.view(np.uint64)
        return np.where(b >> np.uint64(63), ~b, b | np.uint64(1 << 63))
    raise TypeError(f"no order keys for {a.dtype}")


def integral_image(image, square=False, bits=32) -> np.ndarray:
    """integral_image / integral_squared_image (src/integral_image.rs:98-153) of a
    (H, W) or (H, W, C) u8 image: (H+1, W+1[, C]) of u32 (wrapping) or u64."""
    a = np.ascontiguousarray(image, dtype=np.uint8)
    H, W = a.shape[:2]
    C = 1 if a.ndim == 2 else a.shape[2]
    dt = np.uint32 if bits == 32 else np.uint64
    out = np.empty((H + 1, W + 1, C), dt)
    f = lib().nxo_integral_u32 if bits == 32 else lib().nxo_integral_u64
    f(_p(a), W, H, C, int(bool(square)), _p(out))
    return out[:, :, 0] if a.ndim == 2 else out


def suppress_non_maximum(image, radius, naive=False) -> np.ndarray:
    """suppress_non_maximum (src/suppress.rs:10-107); naive=True follows the
    reference tests' own definition (:274-318)."""
    a = np.ascontiguousarray(image)
    H, W = a.shape
    keys = np.ascontiguousarray(order_keys(a))
    keep = np.zeros((H, W), np.uint8)
    f = lib().nxo_suppress_non_maximum_naive if naive else lib().nxo_suppress_non_maximum
    if H and W:
        f(_p(keys), W, H, int(radius), _p(keep))
    return np.where(keep.astype(bool), a, np.zeros((), a.dtype)).astype(a.dtype)


def local_maxima(xs, ys, scores, radius) -> list[int]:
    """local_maxima (src/suppress.rs:111-173): input indices of the kept points in
    the reference's output order."""
    xs = np.ascontiguousarray(xs, np.uint32)
    ys = np.ascontiguousarray(ys, np.uint32)
    sc = np.ascontiguousarray(scores, np.float32)
    out = np.empty(max(len(xs), 1), np.uint32)
    n = lib().nxo_local_maxima(_p(xs), _p(ys), _p(sc), len(xs), int(radius), _p(out))
    return [int(i) for i in out[:n]]


FILTER_OUT = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.int16): 5, np.dtype(np.int32): 6,
              np.dtype(np.float32): 8}


def filter_clamped(image, kernel, out_dtype) -> np.ndarray:
    """filter_clamped (src/filter/mod.rs:29-70, :202-212) of an (H, W) or (H, W, C)
    u8 image by a 2-D f32 or i32 kernel, clamped to out_dtype."""
    a = np.ascontiguousarray(image, np.uint8)
    k = np.ascontiguousarray(kernel)
    H, W = a.shape[:2]
    ch = 1 if a.ndim == 2 else a.shape[2]
    kt = 0 if k.dtype == np.float32 else 1
    od = np.dtype(out_dtype)
    out = np.zeros(a.shape, od)
    lib().nxo_filter_clamped(_p(a), W, H, ch, _p(k), kt, k.shape[1], k.shape[0], FILTER_OUT[od], _p(out))
    return out


# ---- the example workflow: examples/template_matching.rs -------------------------

def convert_to_gray_image(scores) -> np.ndarray:
    """convert_to_gray_image (examples/template_matching.rs:63-76): lo and hi scanned
    with `<` / `>` from +inf / -inf (NaN never an extreme), then
    `(255.0 * (x - lo) / range) as u8` in f32 with Rust's saturating cast."""
    a = np.asarray(scores, np.float32)
    finite = a[~np.isnan(a)]
    lo = finite.min() if finite.size else np.float32(np.inf)
    hi = finite.max() if finite.size else np.float32(-np.inf)
    rng = np.float32(hi - lo)
    with np.errstate(all="ignore"):
        s = (np.float32(255.0) * (a - np.float32(lo))) / rng
        return np.where(np.isnan(s), 0, np.clip(np.trunc(s), 0, 255)).astype(np.uint8)


def draw_green_rect(gray, left, top, width, height) -> np.ndarray:
    """draw_green_rect (examples/template_matching.rs:94-98): the gray image as RGB
    with the outline of Rect::at(left, top).of_size(width, height) in (0, 255, 0):
    draw_hollow_rect_mut (src/drawing/rect.rs:22-35) draws the four edges, each
    an axis-aligned line segment whose pixels outside the image are skipped
    (src/drawing/line.rs:183-200)."""
    g = np.asarray(gray, np.uint8)
    H, W = g.shape
    rgb = np.repeat(g[:, :, None], 3, axis=2)
    right, bottom = left + width - 1, top + height - 1
    green = np.array([0, 255, 0], np.uint8)
    xs = range(max(left, 0), min(right, W - 1) + 1)
    ys = range(max(top, 0), min(bottom, H - 1) + 1)
    for yy in (top, bottom):
        if 0 <= yy < H:
            for xx in xs:
                rgb[yy, xx] = green
    for xx in (left, right):
        if 0 <= xx < W:
            for yy in ys:
                rgb[yy, xx] = green
    return rgb


def template_matching_example(image, x, y, w, h, precision=0) -> dict:
    """What examples/template_matching.rs main (:136-190) computes after decoding:
    the template, the outlined image and the two outlined, rescaled, padded
    score maps (run_match_template :100-134), with the oracle's scores at the
    given precision (0 exact FP64, 1 exact f32, 2 the reference's f32)."""
    a = np.ascontiguousarray(image, np.uint8)
    H, W = a.shape
    assert x + w < W and y + h < H, "invalid sub-image"
    template = a[y:y + h, x:x + w].copy()
    out = {"template": template, "image": draw_green_rect(a, x, y, w, h)}
    for name, method in (("result_sse", 0), ("result_sse_norm", 1)):
        scores = (match_reference(a, template, method) if precision == 2
                  else match_exact(a, template, method, precision=precision))
        scaled = convert_to_gray_image(scores)
        padded = np.zeros((H, W), np.uint8)
        padded[h // 2:h // 2 + scaled.shape[0], w // 2:w // 2 + scaled.shape[1]] = scaled
        out[name] = draw_green_rect(padded, x, y, w, h)
    return out


# ---- the proposal network (learned_oracle.c) ------------------------------------

class _LoParams(C.Structure):
    _fields_ = [("W", C.c_void_p * 5), ("b", C.c_void_p * 5), ("alpha", C.c_double)]


class _LoGrads(C.Structure):
    _fields_ = [("dW", C.c_void_p * 5), ("db", C.c_void_p * 5)]


_LO_SHAPES = [(32, 1, 3, 3)] + [(32, 32, 3, 3)] * 4


def _lo_split(params):
    """Parameter vector (the library's layout) -> lists of FP64 weights and biases."""
    p = np.asarray(params, np.float64)
    Ws, bs, off = [], [], 0
    for shp in _LO_SHAPES:
        n = int(np.prod(shp))
        Ws.append(np.ascontiguousarray(p[off:off + n].reshape(shp)))
        off += n
        bs.append(np.ascontiguousarray(p[off:off + 32]))
        off += 32
    assert off == p.size
    return Ws, bs


def learned_loss_grad(params, scenes, templates, positives, bf16=True, alpha=0.125, want_logits=False):
    """FP64 loss and gradients of the proposal network (learned_oracle.c):
    scenes (n, h, w) u8, templates (t, 48, 48) u8, positives (t,) flat indices.
    Returns (loss, grads in the parameter layout[, logits (t, n*h/4*w/4)])."""
    L = lib()
    if not getattr(L, "_lo_bound", False):
        L.lo_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                   C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.lo_loss_grad.restype = C.c_double
        L._lo_bound = True
    scenes = np.ascontiguousarray(scenes, np.uint8)
    templates = np.ascontiguousarray(templates, np.uint8)
    pos = np.ascontiguousarray(positives, np.int64)
    n, h, w = scenes.shape
    t = templates.shape[0]
    Ws, bs = _lo_split(params)
    P = _LoParams()
    for k in range(5):
        P.W[k] = Ws[k].ctypes.data
        P.b[k] = bs[k].ctypes.data
    P.alpha = alpha
    dW = [np.zeros_like(x) for x in Ws]
    db = [np.zeros_like(x) for x in bs]
    G = _LoGrads()
    for k in range(5):
        G.dW[k] = dW[k].ctypes.data
        G.db[k] = db[k].ctypes.data
    z = np.empty((t, n * (h // 4) * (w // 4)), np.float64) if want_logits else None
    loss = L.lo_loss_grad(C.byref(P), _p(scenes), n, h, w, _p(templates), t, _p(pos), int(bf16), C.byref(G),
                          _p(z))
    grads = np.concatenate([np.concatenate([dW[k].reshape(-1), db[k]]) for k in range(5)])
    return (loss, grads, z) if want_logits else (loss, grads)


def learned_features(params, images, bf16=True, alpha=0.125):
    """FP64 trunk features (learned_oracle.c lo_trunk_forward) of n u8 images
    (n, h, w), sides multiples of 4: an (n, 32, h/4, w/4) array."""
    L = lib()
    if not getattr(L, "_lo_fwd_bound", False):
        L.lo_trunk_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p]
        L.lo_trunk_forward.restype = None
        L._lo_fwd_bound = True
    images = np.ascontiguousarray(images, np.uint8)
    n, h, w = images.shape
    Ws, bs = _lo_split(params)
    P = _LoParams()
    for k in range(5):
        P.W[k] = Ws[k].ctypes.data
        P.b[k] = bs[k].ctypes.data
    P.alpha = alpha
    F = np.empty((n, 32, h // 4, w // 4), np.float64)
    L.lo_trunk_forward(C.byref(P), _p(images), n, h, w, int(bf16), _p(F), None)
    return F
