"""Integral images, non-maximum suppression and filter_clamped on the GPU
against the oracle (src/integral_image.rs, src/suppress.rs,
src/filter/mod.rs). Bar: bit-exact tables and outputs, identical point
lists."""

import json
from pathlib import Path

import numpy as np
import pytest

from imageproc_b200 import filter as fl
from imageproc_b200 import integral_image as ii
from imageproc_b200 import suppress as sp
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_next_tests.json").read_text())


def case(section, name):
    return next(c for c in GOLDEN[section]["cases"] if c["name"] == name)


# ---- integral images ------------------------------------------------------------

SHAPES = [(2, 3), (1, 1), (7, 1), (1, 9), (37, 53), (256, 300), (513, 1031), (1080, 1920)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("channels", [1, 3, 4])
def test_integral_tables_bit_exact(shape, channels):
    g = np.random.default_rng(shape[0] * 7 + channels)
    img = g.integers(0, 256, shape if channels == 1 else shape + (channels,), dtype=np.uint8)
    for square in (False, True):
        for dtype, bits in ((np.uint32, 32), (np.uint64, 64)):
            fn = ii.integral_squared_image if square else ii.integral_image
            got = fn(img, dtype)
            assert np.array_equal(got, O.integral_image(img, square=square, bits=bits)), (square, bits)


def test_integral_golden_and_empty():
    for name in ("test_integral_image_gray", "test_integral_squared_image_gray", "test_integral_image_rgb"):
        c = case("integral_image", name)
        img = np.array(c["image"]["rows"], np.uint8)
        fn = ii.integral_squared_image if c["square"] else ii.integral_image
        assert np.array_equal(fn(img), np.array(c["expected"]["rows"], np.uint32))
    for W, H in ((0, 5), (4, 0), (0, 0)):
        t = ii.integral_image(np.zeros((H, W), np.uint8))
        assert t.shape == (H + 1, W + 1) and not t.any()


def test_integral_u32_wraps_like_the_reference():
    img = np.full((4100, 4100), 255, np.uint8)  # sum of squares > 2^32
    got = ii.integral_squared_image(img, np.uint32)
    exact = ii.integral_squared_image(img, np.uint64)
    assert int(exact[-1, -1]) > 2**32
    assert np.array_equal(got, (exact & 0xFFFFFFFF).astype(np.uint32))


def test_integral_device_form():
    import ctypes as C

    import torch

    from imageproc_b200 import _lib
    g = np.random.default_rng(1)
    img = g.integers(0, 256, (123, 77, 3), dtype=np.uint8)
    d_img = torch.from_numpy(img).cuda()
    d_out = torch.empty((124, 78, 3), dtype=torch.int64, device="cuda")
    L = _lib.lib()
    L.ipb_integral_image_device.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int,
                                            C.c_void_p, C.c_void_p]
    L.ipb_integral_image_device.restype = C.c_int
    _lib.check(L.ipb_integral_image_device(d_img.data_ptr(), 77, 123, 3, 1, 64, d_out.data_ptr(),
                                           torch.cuda.current_stream().cuda_stream or None))
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy().view(np.uint64), O.integral_image(img, square=True, bits=64))
    # Luma: the tiled one-write path, whose carries live in the context's
    # scratch; two calls in a row on one stream share it
    stream = torch.cuda.current_stream().cuda_stream or None
    for H, W in ((300, 512), (1000, 777), (33, 8)):
        gray = g.integers(0, 256, (H, W), dtype=np.uint8)
        d_gray = torch.from_numpy(gray).cuda()
        d32 = torch.empty((H + 1, W + 1), dtype=torch.int32, device="cuda")
        d64 = torch.empty((H + 1, W + 1), dtype=torch.int64, device="cuda")
        _lib.check(L.ipb_integral_image_device(d_gray.data_ptr(), W, H, 1, 1, 32, d32.data_ptr(), stream))
        _lib.check(L.ipb_integral_image_device(d_gray.data_ptr(), W, H, 1, 0, 64, d64.data_ptr(), stream))
        torch.cuda.synchronize()
        assert np.array_equal(d32.cpu().numpy().view(np.uint32), O.integral_image(gray, square=True, bits=32))
        assert np.array_equal(d64.cpu().numpy().view(np.uint64), O.integral_image(gray, square=False, bits=64))


# ---- suppress_non_maximum ---------------------------------------------------------

DTYPES = [np.uint8, np.uint16, np.uint32, np.uint64, np.int8, np.int16, np.int32, np.int64, np.float32]


@pytest.mark.parametrize("dtype", DTYPES)
def test_suppress_matches_oracle_with_ties(dtype):
    g = np.random.default_rng(np.dtype(dtype).num)
    signed = np.dtype(dtype).kind in "if"
    for _ in range(40):
        H, W = int(g.integers(1, 40)), int(g.integers(1, 40))
        a = g.integers(-4 if signed else 0, 5, (H, W)).astype(dtype)  # few values: many ties
        r = int(g.integers(0, 9))
        assert np.array_equal(sp.suppress_non_maximum(a, r), O.suppress_non_maximum(a, r)), (H, W, r)


@pytest.mark.parametrize("dtype", [np.uint8, np.int32, np.uint64, np.float32])
def test_suppress_full_range_values(dtype):
    g = np.random.default_rng(3)
    info = np.finfo(dtype) if np.dtype(dtype).kind == "f" else np.iinfo(dtype)
    if np.dtype(dtype).kind == "f":
        a = g.standard_normal((300, 500)).astype(dtype) * 1e3
        a[0, :5] = [0.0, -0.0, np.inf, -np.inf, np.nan]
    else:
        a = g.integers(info.min, info.max, (300, 500), dtype=dtype, endpoint=True)
    for r in (1, 3, 16):
        got = sp.suppress_non_maximum(a, r)
        exp = O.suppress_non_maximum(a, r)
        assert np.array_equal(got.view(np.uint8), exp.view(np.uint8)), r


def test_suppress_golden_and_edges():
    c = case("suppress", "test_suppress_non_maximum")
    W, H = c["size"]
    img = np.zeros((H, W), np.uint8)
    for x, y, v in c["pixels"]:
        img[y, x] = v
    exp = np.zeros((H, W), np.uint8)
    for x, y, v in c["expected"]:
        exp[y, x] = v
    assert np.array_equal(sp.suppress_non_maximum(img, c["radius"]), exp)
    c = case("suppress", "test_suppress_non_maximum_handles_radius_greater_than_image_side")
    for W, H in c["sizes"]:
        a = np.random.default_rng(W).integers(0, 3, (H, W)).astype(np.uint8)
        assert np.array_equal(sp.suppress_non_maximum(a, c["radius"]), O.suppress_non_maximum(a, c["radius"]))
    assert sp.suppress_non_maximum(np.zeros((0, 5), np.uint8), 3).shape == (0, 5)


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.float32])
def test_suppress_one_pass_tiles_and_two_pass_radii(dtype):
    # radii 0..16 take the one-pass tile kernel (128 x 32 tiles, so these maps
    # cross tile edges in both directions); 17 and 40 the two-pass kernels
    g = np.random.default_rng(21)
    for r in (0, 1, 4, 5, 8, 9, 12, 16, 17, 40):
        H, W = int(g.integers(33, 200)), int(g.integers(129, 420))
        a = g.integers(0, 7, (H, W)).astype(dtype)  # many ties across tiles
        assert np.array_equal(sp.suppress_non_maximum(a, r), O.suppress_non_maximum(a, r)), (H, W, r)


def test_suppress_device_in_place():
    # an output that is the image itself runs the two-pass kernels, which read
    # each pixel only where they write it
    import ctypes as C

    import torch

    from imageproc_b200 import _lib
    L = _lib.lib()
    L.ipb_suppress_non_maximum_f32_device.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                                      C.c_void_p, C.c_void_p]
    L.ipb_suppress_non_maximum_f32_device.restype = C.c_int
    g = np.random.default_rng(22)
    a = g.standard_normal((97, 300)).astype(np.float32)
    exp = O.suppress_non_maximum(a, 6)
    d = torch.from_numpy(a).cuda()
    stream = torch.cuda.current_stream().cuda_stream or None
    _lib.check(L.ipb_suppress_non_maximum_f32_device(d.data_ptr(), 300, 97, 6, d.data_ptr(), stream))
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), exp.view(np.uint32))


def test_suppress_wide_radius_and_large_image():
    g = np.random.default_rng(11)
    a = g.integers(0, 6, (50, 40)).astype(np.uint16)
    assert np.array_equal(sp.suppress_non_maximum(a, 3000), O.suppress_non_maximum(a, 3000))  # global-memory rows
    b = g.integers(0, 50, (1080, 1920)).astype(np.uint8)
    assert np.array_equal(sp.suppress_non_maximum(b, 5), O.suppress_non_maximum(b, 5))


# ---- local_maxima -------------------------------------------------------------------

def test_local_maxima_golden():
    c = case("suppress", "test_local_maxima")
    pts = [tuple(p) for p in c["points"]]
    assert [list(p) for p in sp.local_maxima(pts, c["radius"])] == c["expected"]
    assert sp.local_maxima([], 3) == []


def test_local_maxima_matches_oracle():
    g = np.random.default_rng(5)
    for trial in range(60):
        n = int(g.integers(1, 400))
        span = int(g.integers(1, 60))
        xs = g.integers(0, span, n).astype(np.uint32)
        ys = g.integers(0, span, n).astype(np.uint32)
        sc = g.integers(0, 6, n).astype(np.float32)  # ties and duplicate positions
        if trial % 5 == 0:
            sc[g.integers(0, n, 3)] = np.nan
        r = int(g.integers(0, 8))
        assert sp.local_maxima_indices(xs, ys, sc, r) == O.local_maxima(xs, ys, sc, r), trial


# ---- filter_clamped -----------------------------------------------------------------

F32_OUTS = [np.uint8, np.uint16, np.float32]
I32_OUTS = [np.uint8, np.uint16, np.int16, np.int32]


def _same(got, exp):
    # bit-exact, except that a NaN is any NaN: the GPU writes its canonical NaN
    # where x86 propagates the kernel's NaN payload
    if got.dtype == np.float32:
        nan = np.isnan(exp)
        return np.array_equal(np.isnan(got), nan) and np.array_equal(got[~nan].view(np.uint32),
                                                                      exp[~nan].view(np.uint32))
    return np.array_equal(got, exp)


@pytest.mark.parametrize("channels", [1, 3, 4])
def test_filter_clamped_matches_oracle(channels):
    g = np.random.default_rng(channels)
    for trial in range(24):
        H, W = int(g.integers(1, 70)), int(g.integers(1, 90))
        img = g.integers(0, 256, (H, W) if channels == 1 else (H, W, channels), dtype=np.uint8)
        kh, kw = int(g.integers(1, 9)), int(g.integers(1, 9))  # even and odd sides, some wider than the image
        if trial % 2:
            k = (g.standard_normal((kh, kw)) * 3).astype(np.float32)
            if trial % 6 == 1:
                k[0, 0] = np.nan
            outs = F32_OUTS
        else:
            k = g.integers(-2**20, 2**20, (kh, kw)).astype(np.int32)  # sums wrap in i32
            outs = I32_OUTS
        for od in outs:
            got = fl.filter_clamped(img, k, od)
            exp = O.filter_clamped(img, k, od)
            assert _same(got, exp), (trial, od, kh, kw)


def test_filter_large_kernel_and_image():
    g = np.random.default_rng(9)
    img = g.integers(0, 256, (300, 420), dtype=np.uint8)
    k = g.random((3, 70), dtype=np.float32) / 100  # wider than the shared-memory tile path takes
    assert np.array_equal(fl.filter_clamped(img, k, np.float32).view(np.uint32),
                          O.filter_clamped(img, k, np.float32).view(np.uint32))
    big = g.integers(0, 256, (1080, 1920), dtype=np.uint8)
    k5 = g.random((5, 5), dtype=np.float32) / 5
    assert np.array_equal(fl.filter_clamped(big, k5, np.uint8), O.filter_clamped(big, k5, np.uint8))


def test_filter_golden_and_forms():
    for c in GOLDEN["filter"]["cases"]:
        img = np.array(c["image"]["rows"], np.uint8)
        exp = np.array(c["expected"]["rows"])
        if c.get("separable"):
            k = (np.full(c["taps"], np.float32(1) / np.float32(c["kernel_one_over"]), np.float32)
                 if c["kernel_type"] == "f32" else np.full(c["taps"], c["kernel_value"], np.int32))
            got = fl.separable_filter_equal(img, k)
        elif c["kernel_type"] == "i32":
            k = np.array(c["kernel"], np.int32).reshape(c["kernel_height"], c["kernel_width"])
            got = fl.filter_clamped(img, k, np.int16)
        else:
            k = np.full(3, np.float32(1) / np.float32(c["kernel_one_over"]), np.float32)
            got = fl.horizontal_filter(img, k) if c["kernel_height"] == 1 else fl.vertical_filter(img, k)
        assert np.array_equal(got, exp), c["name"]
    img = np.array([[1, 2, 3], [4, 5, 6], [7, 8, 9]], np.uint8)
    assert np.array_equal(fl.laplacian_filter(img), O.filter_clamped(img, fl.LAPLACIAN, np.int16))
    with pytest.raises(fl.Panic, match="^width and height must be non-zero$"):
        fl.filter_clamped(img, np.zeros((0, 3), np.float32))
    with pytest.raises(fl.Panic, match="^the two 1D kernels must be the same length$"):
        fl.separable_filter(img, np.ones(3, np.float32), np.ones(5, np.float32))
    with pytest.raises(ValueError):
        fl.filter_clamped(img, np.ones((3, 3), np.float32), np.int16)  # no Clamp<f32> for i16
