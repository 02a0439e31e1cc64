"""The CPU oracle against the reference's own known-answer tests.

Pins the oracle (src/template_matching.rs:518-833 as extracted into
tests/golden/reference_unit_tests.json) before it is trusted as the checker
of the CUDA path, and cross-checks its flavours against an independent numpy
restatement on small random cases.
"""

import numpy as np
import pytest

from conftest import f32_bits, gray
from oracle import oracle as O


def _case_inputs(c):
    img = gray(c["image"]["rows"])
    tpl = gray(c["template"]["rows"])
    mask = gray(c["mask"]["rows"]) if "mask" in c else None
    return img, tpl, mask


def _match_cases(cases, panics=False):
    return [c for c in cases if c["kind"] != "find_extremes" and c["should_panic"] == panics]


def ulp_diff(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def test_golden_file_covers_reference_tests(golden_cases):
    names = {c["name"] for c in golden_cases}
    assert len(golden_cases) == 13
    assert "test_find_extremes" in names
    assert sum(c["should_panic"] for c in golden_cases) == 2


def test_reference_restatement_is_bit_exact_on_goldens(golden_cases):
    for c in _match_cases(golden_cases):
        img, tpl, mask = _case_inputs(c)
        got = O.match_reference(img, tpl, c["method"], mask, threads=1)
        exp = f32_bits(c["expected"]["bits"])
        assert got.view(np.uint32).tolist() == exp.view(np.uint32).tolist(), c["name"]


def test_exact_sums_with_f32_normalisation_are_bit_exact_on_goldens(golden_cases):
    for c in _match_cases(golden_cases):
        img, tpl, mask = _case_inputs(c)
        got = O.match_exact(img, tpl, c["method"], mask, precision=1)
        exp = f32_bits(c["expected"]["bits"])
        assert got.view(np.uint32).tolist() == exp.view(np.uint32).tolist(), c["name"]


def test_fp64_normalisation_within_one_ulp_of_goldens(golden_cases):
    worst = 0
    for c in _match_cases(golden_cases):
        img, tpl, mask = _case_inputs(c)
        got = O.match_exact(img, tpl, c["method"], mask, precision=0)
        d = ulp_diff(got, f32_bits(c["expected"]["bits"]))
        worst = max(worst, int(d.max()))
        if c["method"] in (0, 2):  # unnormalised scores are exact integers
            assert d.max() == 0, c["name"]
    assert worst <= 1


def test_panic_cases_fail_in_the_oracle(golden_cases):
    for c in _match_cases(golden_cases, panics=True):
        img, tpl, _ = _case_inputs(c)
        with pytest.raises(O.OracleError):
            O.match_reference(img, tpl, c["method"])


def test_find_extremes_golden(golden_cases):
    c = next(c for c in golden_cases if c["kind"] == "find_extremes")
    mx, mn, mxl, mnl = O.find_extremes(gray(c["image"]["rows"]))
    e = c["expected"]
    assert (mx, mn, list(mxl), list(mnl)) == (e["max_value"], e["min_value"],
                                              e["max_value_location"], e["min_value_location"])


# ---- independent numpy restatement (tiny sizes) ---------------------------

def numpy_reference(img, tpl, method, mask=None):
    """Sequential f32 scores with numpy scalars, written from the reference's
    closures (src/template_matching.rs:219-375)."""
    f = np.float32
    H, W = img.shape
    h, w = tpl.shape
    out = np.zeros((H - h + 1, W - w + 1), np.float32)
    if mask is None:
        tss = f(0)
        for v in tpl.reshape(-1):
            tss = f(tss + f(f(v) * f(v)))
    else:
        tss = f(0)
        for v, m in zip(tpl.reshape(-1), mask.reshape(-1)):
            p = f(f(v) * f(m))
            tss = f(tss + f(p * p))
    for y in range(H - h + 1):
        for x in range(W - w + 1):
            s = f(0)
            q = f(0)
            for dy in range(h):
                for dx in range(w):
                    i, t = f(img[y + dy, x + dx]), f(tpl[dy, dx])
                    m = f(mask[dy, dx]) if mask is not None else None
                    if mask is None:
                        if method in (0, 1):
                            d = f(t - i)
                            s = f(s + f(d * d))
                        else:
                            s = f(s + f(i * t))
                        q = f(q + f(i * i))
                    else:
                        if method in (0, 1):
                            e = f(f(t - i) * m)
                            s = f(s + f(e * e))
                        else:
                            s = f(s + f(f(f(t * i) * m) * m))
                        p = f(i * m)
                        q = f(q + f(p * p))
            if method in (1, 3):
                n = np.sqrt(f(q * tss) if mask is None else f(tss * q), dtype=np.float32)
                s = f(s / n) if n > 0 else s
            out[y, x] = s
    return out


@pytest.mark.parametrize("seed", range(6))
def test_oracle_flavours_agree_with_numpy_restatement(seed):
    g = np.random.default_rng(seed)
    H, W = g.integers(3, 9, size=2)
    h, w = g.integers(1, min(H, W) + 1, size=2)
    img = g.integers(0, 256, (H, W), dtype=np.uint8)
    tpl = g.integers(0, 256, (h, w), dtype=np.uint8)
    for mask in (None, g.integers(0, 2, (h, w), dtype=np.uint8),
                 g.integers(0, 256, (h, w), dtype=np.uint8)):
        for method in range(4):
            ref = O.match_reference(img, tpl, method, mask, threads=2)
            np.testing.assert_array_equal(ref.view(np.uint32),
                                          numpy_reference(img, tpl, method, mask).view(np.uint32))
        # exact integer sums against numpy
        X, Y, tss = O.sums(img, tpl, mask)
        m = np.ones_like(tpl) if mask is None else mask
        U = tpl.astype(np.uint64) * m * m
        V = m.astype(np.uint64) ** 2
        for y in range(H - h + 1):
            for x in range(W - w + 1):
                win = img[y:y + h, x:x + w].astype(np.uint64)
                assert X[y, x] == (win * U).sum()
                assert Y[y, x] == (win * win * V).sum()
        assert tss == ((tpl.astype(np.uint64) * m) ** 2).sum()


def test_reference_equals_exact_f32_when_reference_sums_are_exact():
    # unmasked templates of <= 258 pixels keep every f32 partial sum exact
    g = np.random.default_rng(7)
    img = g.integers(0, 256, (40, 50), dtype=np.uint8)
    tpl = g.integers(0, 256, (16, 16), dtype=np.uint8)
    for method in range(4):
        ref = O.match_reference(img, tpl, method)
        ex = O.match_exact(img, tpl, method, precision=1)
        np.testing.assert_array_equal(ref.view(np.uint32), ex.view(np.uint32))


def test_reference_rounds_on_large_templates():
    # 64x64 unmasked SSE exceeds 2^24, so the reference's own f32 sums round
    g = np.random.default_rng(8)
    img = g.integers(0, 256, (70, 70), dtype=np.uint8)
    tpl = g.integers(0, 256, (64, 64), dtype=np.uint8)
    ref = O.match_reference(img, tpl, 0)
    ex = O.match_exact(img, tpl, 0, precision=0)
    assert (ref != ex).any()
    rel = np.abs(ref.astype(np.float64) - ex.astype(np.float64)) / ex.astype(np.float64)
    assert rel.max() < 2e-4  # sequential f32 drift over 4096 terms
