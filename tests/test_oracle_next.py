"""The oracle for integral images and non-maximum suppression against the
reference's known-answer tests (src/integral_image.rs:471-567,
src/suppress.rs:209-270), extracted as text into
tests/golden/reference_next_tests.json, and against the naive definition of
suppress_non_maximum the reference's own tests hold (src/suppress.rs:274-318).
No GPU needed."""

import json
from pathlib import Path

import numpy as np
import pytest

from imageproc_b200 import integral_image as ii
from oracle import oracle as O

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_next_tests.json").read_text())


def as_array(img):
    return np.array(img["rows"], dtype=np.uint32 if img["type"] == "u32" else np.uint8)


def case(section, name):
    return next(c for c in GOLDEN[section]["cases"] if c["name"] == name)


@pytest.mark.parametrize("name", ["test_integral_image_gray", "test_integral_squared_image_gray",
                                  "test_integral_image_rgb"])
def test_integral_tables(name):
    c = case("integral_image", name)
    got = O.integral_image(as_array(c["image"]), square=c["square"], bits=32)
    assert np.array_equal(got, as_array(c["expected"]))
    got64 = O.integral_image(as_array(c["image"]), square=c["square"], bits=64)
    assert np.array_equal(got64, as_array(c["expected"]).astype(np.uint64))


@pytest.mark.parametrize("name", ["test_sum_image_pixels", "test_sum_image_pixels_rgb"])
def test_sum_image_pixels(name):
    c = case("integral_image", name)
    table = O.integral_image(as_array(c["image"]), bits=32)
    assert len(c["sums"]) == 9
    for s in c["sums"]:
        assert ii.sum_image_pixels(table, *s["ltrb"]).tolist() == s["expected"]


def test_variance_doc_example():
    # the example of src/integral_image.rs:283-300: right two columns of [1 2 3; 4 5 6]
    img = np.array([[1, 2, 3], [4, 5, 6]], np.uint8)
    vals = np.array([2.0, 3.0, 5.0, 6.0])
    var = float(((vals - vals.mean()) ** 2).sum() / 4)
    got = ii.variance(O.integral_image(img), O.integral_image(img, square=True), 1, 0, 2, 1)
    assert got == var


def test_u32_tables_wrap():
    img = np.full((300, 300), 255, np.uint8)
    t32 = O.integral_image(img, square=True, bits=32)
    t64 = O.integral_image(img, square=True, bits=64)
    assert t64[-1, -1] == 300 * 300 * 255 * 255 > 2**32
    assert np.array_equal(t32, (t64 & 0xFFFFFFFF).astype(np.uint32))


def test_suppress_golden():
    c = case("suppress", "test_suppress_non_maximum")
    W, H = c["size"]
    img = np.zeros((H, W), np.uint8)
    for x, y, v in c["pixels"]:
        img[y, x] = v
    exp = np.zeros((H, W), np.uint8)
    for x, y, v in c["expected"]:
        exp[y, x] = v
    assert np.array_equal(O.suppress_non_maximum(img, c["radius"]), exp)
    assert np.array_equal(O.suppress_non_maximum(img, c["radius"], naive=True), exp)


def test_suppress_radius_greater_than_side():
    c = case("suppress", "test_suppress_non_maximum_handles_radius_greater_than_image_side")
    for W, H in c["sizes"]:
        assert O.suppress_non_maximum(np.zeros((H, W), np.uint8), c["radius"]).shape == (H, W)


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.uint32, np.int64, np.float32])
def test_suppress_block_algorithm_equals_naive(dtype):
    # the reference's proptest (src/suppress.rs:338-346) at radius 3, widened
    g = np.random.default_rng(7)
    for _ in range(200):
        a = g.integers(-3 if np.dtype(dtype).kind in "if" else 0, 4,
                       (int(g.integers(0, 12)), int(g.integers(0, 12)))).astype(dtype)
        r = int(g.integers(0, 7))
        assert np.array_equal(O.suppress_non_maximum(a, r), O.suppress_non_maximum(a, r, naive=True))


def test_local_maxima_golden():
    c = case("suppress", "test_local_maxima")
    pts = c["points"]
    idx = O.local_maxima([p[0] for p in pts], [p[1] for p in pts], [p[2] for p in pts], c["radius"])
    assert [pts[i] for i in idx] == c["expected"]


# ---- filter_clamped (src/filter/mod.rs) -------------------------------------

def golden_kernel(c):
    if c["kernel_type"] == "i32":
        if "kernel" in c:
            return np.array(c["kernel"], np.int32).reshape(c["kernel_height"], c["kernel_width"])
        return np.full(c["taps"], c["kernel_value"], np.int32)
    k = np.float32(1) / np.float32(c["kernel_one_over"])
    if c.get("separable"):
        return np.full(c["taps"], k, np.float32)
    return np.full((c["kernel_height"], c["kernel_width"]), k, np.float32)


def oracle_golden_filter(c):
    img = np.array(c["image"]["rows"], np.uint8)
    k = golden_kernel(c)
    if c.get("separable"):
        h = O.filter_clamped(img, k.reshape(1, -1), np.uint8)
        return O.filter_clamped(h, k.reshape(-1, 1), np.uint8)
    od = {"i16": np.int16, "u8": np.uint8}[c["expected"]["type"]]
    return O.filter_clamped(img, k, od)


@pytest.mark.parametrize("name", [c["name"] for c in GOLDEN["filter"]["cases"]])
def test_filter_golden(name):
    c = case("filter", name)
    exp = np.array(c["expected"]["rows"])
    assert np.array_equal(oracle_golden_filter(c), exp)


def test_filter_clamp_rules():
    img = np.array([[10, 20], [30, 40]], np.uint8)
    # NaN accumulators clamp to the maximum, negatives to the minimum
    k = np.array([[np.nan]], np.float32)
    assert (O.filter_clamped(img, k, np.uint8) == 255).all()
    assert (O.filter_clamped(img, -np.ones((1, 1), np.float32), np.uint16) == 0).all()
    big = np.full((1, 1), 2**30, np.int32)  # wraps in i32, then clamps
    got = O.filter_clamped(img, big, np.int32)
    assert got[0, 0] == -2**31  # 10 * 2^30 = 2^33 + 2^31 wraps to 2^31, i.e. -2^31 as i32
