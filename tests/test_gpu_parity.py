"""Parity of the CUDA path with the oracle, through the C ABI.

Bar: bit-exact. EXACT_FP64 and EXACT_F32 scores equal the oracle's
exact-sum epilogue bit for bit; REFERENCE_F32 scores equal the reference's
f32 arithmetic bit for bit; unnormalised scores are exact integers rounded
once to f32. Against the reference's own goldens EXACT_FP64 is within 1 ulp
(tolerance: 1 ulp, the reference rounds its normalisation in f32).
"""

import numpy as np
import pytest

from conftest import f32_bits, gray
from imageproc_b200 import synthetic
from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P = tm.Precision
M = tm.MatchTemplateMethod


@pytest.fixture(autouse=True)
def _restore_precision():
    old = tm.get_precision()
    yield
    tm.set_precision(old)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def ulps(a, b):
    return np.abs(bits(a).view(np.int32).astype(np.int64) - bits(b).view(np.int32).astype(np.int64))


def gpu(image, template, method, mask=None, precision=P.ExactFp64, parallel=False):
    tm.set_precision(precision)
    if mask is None:
        fn = tm.match_template_parallel if parallel else tm.match_template
        return fn(image, template, method)
    fn = tm.match_template_with_mask_parallel if parallel else tm.match_template_with_mask
    return fn(image, template, method, mask)


def oracle_for(image, template, method, mask, precision):
    if precision == P.ReferenceF32:
        return O.match_reference(image, template, method, mask)
    return O.match_exact(image, template, method, mask, precision=int(precision))


# ---- the reference's known-answer tests -------------------------------------

def test_reference_goldens_all_precisions(golden_cases):
    for c in golden_cases:
        if c["kind"] == "find_extremes" or c["should_panic"]:
            continue
        img, tpl = gray(c["image"]["rows"]), gray(c["template"]["rows"])
        mask = gray(c["mask"]["rows"]) if "mask" in c else None
        exp = f32_bits(c["expected"]["bits"])
        for par in (False, True):
            for prec in (P.ReferenceF32, P.ExactF32):
                got = gpu(img, tpl, c["method"], mask, prec, par)
                assert bits(got).tolist() == bits(exp).tolist(), (c["name"], prec, par)
            got = gpu(img, tpl, c["method"], mask, P.ExactFp64, par)
            assert ulps(got, exp).max() <= 1, c["name"]
            assert bits(got).tolist() == bits(O.match_exact(img, tpl, c["method"], mask, 0)).tolist()


def test_reference_find_extremes_golden(golden_cases):
    c = next(c for c in golden_cases if c["kind"] == "find_extremes")
    e = c["expected"]
    got = tm.find_extremes(gray(c["image"]["rows"]))
    assert got == tm.Extremes(e["max_value"], e["min_value"], tuple(e["max_value_location"]),
                              tuple(e["min_value_location"]))


# ---- random shapes against the oracle ---------------------------------------

def _random_case(seed):
    g = np.random.default_rng(1000 + seed)
    H = int(g.integers(1, 48))
    W = int(g.integers(1, 300))
    h = int(g.integers(1, min(H, 40) + 1))
    w = int(g.integers(1, min(W, 150) + 1))
    img = g.integers(0, 256, (H, W), dtype=np.uint8)
    if seed % 4 == 0:
        img[:] = 255  # saturated: largest sums
    tpl = g.integers(0, 256, (h, w), dtype=np.uint8)
    masks = [None, (g.random((h, w)) < 0.7).astype(np.uint8), g.integers(0, 256, (h, w), dtype=np.uint8)]
    return img, tpl, masks


@pytest.mark.parametrize("seed", range(16))
def test_random_shapes_bit_exact(seed):
    img, tpl, masks = _random_case(seed)
    for mask in masks:
        for method in M:
            for prec in P:
                got = gpu(img, tpl, method, mask, prec)
                exp = oracle_for(img, tpl, method, mask, prec)
                assert got.shape == exp.shape
                bad = np.argwhere(bits(got) != bits(exp))
                assert bad.size == 0, (img.shape, tpl.shape, mask is not None, method, prec,
                                       bad[:3], got[tuple(bad[0])], exp[tuple(bad[0])])


# ---- the workloads at full size ---------------------------------------------

def test_uniform_scene_512_template_16_sse():
    image, template, loc = synthetic.uniform_scene()
    X, Y, tss = O.sums(image, template)
    exact = (Y + np.uint64(tss) - np.uint64(2) * X)
    for prec in P:
        got = gpu(image, template, M.SumOfSquaredErrors, None, prec)
        assert got.shape == (497, 497)
        # 256 template pixels: every f32 partial sum of the reference is exact,
        # so all three precisions equal the exact integer score
        assert bits(got).tolist() == bits(exact.astype(np.float32)).tolist()
        assert np.array_equal(got.astype(np.uint64), exact)
    ex = tm.find_extremes(got)
    assert ex.min_value_location == loc or got[loc[1], loc[0]] == ex.min_value


@pytest.fixture(scope="module")
def blob_scene():
    return synthetic.blob_scene()


@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("method", list(M))
def test_blob_scene_1920x1080_template_64_exact(blob_scene, method, masked):
    image, template, mask, loc = blob_scene
    m = mask if masked else None
    got = gpu(image, template, method, m, P.ExactFp64)
    exp = O.match_exact(image, template, method, m, precision=0)
    assert got.shape == (1017, 1857)
    assert bits(got).tolist() == bits(exp).tolist()
    # against the reference's own f32 arithmetic on a band of rows: report-
    # level bound (the reference's sums over 4096 terms round)
    ref = O.match_reference(image, template, method, m, rows=(500, 508))
    rel = np.abs(got[500:508].astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-30)
    assert rel.max() < 1e-3


@pytest.mark.parametrize("method", list(M))
def test_blob_scene_reference_precision_band(blob_scene, method):
    image, template, mask, _ = blob_scene
    for m in (None, mask):
        got = gpu(image, template, method, m, P.ReferenceF32)
        ref = O.match_reference(image, template, method, m, rows=(0, 6))
        assert bits(got[:6]).tolist() == bits(ref).tolist()
        ref = O.match_reference(image, template, method, m, rows=(1011, 1017))
        assert bits(got[1011:]).tolist() == bits(ref).tolist()


def test_general_mask_full_size(blob_scene):
    image, template, _, _ = blob_scene
    g = np.random.default_rng(3)
    mask = g.integers(0, 256, template.shape, dtype=np.uint8)
    for method in M:
        got = gpu(image[:300, :500], template, method, mask, P.ExactFp64)
        exp = O.match_exact(image[:300, :500], template, method, mask, precision=0)
        assert bits(got).tolist() == bits(exp).tolist()


# ---- edge cases the reference defines ---------------------------------------

def test_template_same_size_as_image():
    g = np.random.default_rng(5)
    img = g.integers(0, 256, (9, 13), dtype=np.uint8)
    for method in M:
        for prec in P:
            got = gpu(img, img, method, None, prec)
            assert got.shape == (1, 1)
            assert bits(got).tolist() == bits(oracle_for(img, img, method, None, prec)).tolist()


@pytest.mark.parametrize("tshape", [(0, 0), (0, 3), (3, 0)])
def test_zero_sized_template_gives_zeros(tshape):
    img = np.full((5, 7), 9, np.uint8)
    tpl = np.zeros(tshape, np.uint8)
    for method in M:
        for prec in P:
            got = gpu(img, tpl, method, None, prec)
            assert got.shape == (5 - tshape[0] + 1, 7 - tshape[1] + 1)
            assert not got.any()
            got = gpu(img, tpl, method, tpl.copy(), prec)
            assert not got.any()


def test_zero_norm_returns_raw_score():
    img = np.zeros((6, 6), np.uint8)
    tpl = np.full((3, 3), 7, np.uint8)
    for prec in P:
        got = gpu(img, tpl, M.SumOfSquaredErrorsNormalized, None, prec)
        assert (got == 9 * 49).all()
        got = gpu(img, tpl, M.CrossCorrelationNormalized, None, prec)
        assert (got == 0).all()


def test_large_saturated_template_is_exact():
    # 300x300 template of 255s: sums far above 2^32, exact in u64
    img = np.full((310, 305), 255, np.uint8)
    img[::7, ::5] = 3
    tpl = np.full((300, 300), 255, np.uint8)
    for method in M:
        got = gpu(img, tpl, method, None, P.ExactFp64)
        exp = O.match_exact(img, tpl, method, None, precision=0)
        assert bits(got).tolist() == bits(exp).tolist()


def test_thin_images():
    g = np.random.default_rng(11)
    for (H, W), (h, w) in [((1, 200), (1, 17)), ((200, 1), (33, 1)), ((1, 1), (1, 1))]:
        img = g.integers(0, 256, (H, W), dtype=np.uint8)
        tpl = g.integers(0, 256, (h, w), dtype=np.uint8)
        for method in M:
            for prec in P:
                got = gpu(img, tpl, method, None, prec)
                assert bits(got).tolist() == bits(oracle_for(img, tpl, method, None, prec)).tolist()


# ---- find_extremes ------------------------------------------------------------

DTYPES = [np.uint8, np.uint16, np.uint32, np.uint64, np.int8, np.int16, np.int32, np.int64,
          np.float32, np.float64]


@pytest.mark.parametrize("dtype", DTYPES)
def test_find_extremes_matches_oracle(dtype):
    g = np.random.default_rng(21)
    for shape in [(1, 1), (3, 5), (257, 1031), (1024, 2049)]:
        if np.issubdtype(dtype, np.floating):
            a = g.standard_normal(shape).astype(dtype)
        else:
            info = np.iinfo(dtype)
            a = g.integers(info.min, info.max, size=shape, dtype=dtype, endpoint=True)
        got = tm.find_extremes(a)
        mx, mn, mxl, mnl = O.find_extremes(a)
        assert (got.max_value, got.min_value, got.max_value_location, got.min_value_location) == \
            (mx, mn, mxl, mnl)


def test_find_extremes_ties_resolve_to_first_pixel():
    a = np.zeros((300, 700), np.float32)
    got = tm.find_extremes(a)
    assert got.max_value_location == (0, 0) and got.min_value_location == (0, 0)
    a[5, 3] = a[200, 1] = a[299, 699] = 2.0
    a[7, 600] = a[100, 5] = -1.0
    got = tm.find_extremes(a)
    assert got.max_value_location == (3, 5) and got.min_value_location == (600, 7)


def test_find_extremes_nan_and_signed_zero_rules():
    a = np.ones((64, 64), np.float32)
    a[3, 3] = np.nan
    a[10, 10] = 5
    got = tm.find_extremes(a)
    assert got.max_value == 5 and got.max_value_location == (10, 10)
    assert got.min_value == 1 and got.min_value_location == (0, 0)
    a[0, 0] = np.nan  # a NaN seed is never replaced
    got = tm.find_extremes(a)
    assert np.isnan(got.max_value) and np.isnan(got.min_value)
    assert got.max_value_location == (0, 0) == got.min_value_location
    b = np.zeros((4, 4), np.float32)
    b[0, 0] = 0.0
    b[2, 2] = -0.0  # equal to +0.0: not smaller, the seed stays
    got = tm.find_extremes(b)
    assert got.min_value_location == (0, 0) and not np.signbit(got.min_value)
    c = np.full((8, 8), np.inf, np.float64)
    c[4, 4] = -np.inf
    got = tm.find_extremes(c)
    assert got.max_value_location == (0, 0) and got.min_value_location == (4, 4)


def test_find_extremes_on_score_map_after_match(blob_scene):
    image, template, _, loc = blob_scene
    scores = gpu(image, template, M.SumOfSquaredErrors)
    got = tm.find_extremes(scores)
    mx, mn, mxl, mnl = O.find_extremes(scores)
    assert (got.min_value, got.min_value_location, got.max_value, got.max_value_location) == \
        (mn, mnl, mx, mxl)


# ---- device-resident API -------------------------------------------------------

def test_device_api_matches_host_api(blob_scene):
    import torch

    from imageproc_b200 import device
    image, template, mask, _ = blob_scene
    di = torch.from_numpy(image).cuda()
    dt = torch.from_numpy(template).cuda()
    dm = torch.from_numpy(mask).cuda()
    for method in M:
        for m, dmask in ((None, None), (mask, dm)):
            host = gpu(image, template, method, m, P.ExactFp64)
            dev = device.match_template_device(di, dt, method, dmask, mask_is_binary=True)
            torch.cuda.synchronize()
            assert bits(dev.cpu().numpy()).tolist() == bits(host).tolist()
    ex = device.find_extremes_device(dev)
    ref = tm.find_extremes(dev.cpu().numpy())
    assert (ex.min_value, ex.min_value_location) == (ref.min_value, ref.min_value_location)
