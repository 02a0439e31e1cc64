"""The oracle's fast exact form (used by the full-size parity checks) against
its plain restatement: same scores, same find_extremes, for every method and
both exact precisions, odd and even widths, template rows of zeros, ties, and
row bands of many templates."""

import numpy as np
import pytest

from oracle import oracle as O


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("W,H,w,h", [(97, 61, 16, 8), (130, 77, 33, 17), (64, 64, 1, 1),
                                      (40, 300, 40, 5), (301, 45, 129, 3), (70, 70, 63, 70)])
@pytest.mark.parametrize("precision", [0, 1])
def test_fast_equals_plain(W, H, w, h, precision):
    rng = np.random.default_rng(W * 1000 + h)
    image = rng.integers(0, 256, size=(H, W), dtype=np.uint8)
    template = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
    template[h // 2] = 0  # a template row of zeros is skipped by the fast loop
    for method in range(4):
        plain = O.match_exact(image, template, method, precision=precision)
        fast, ext = O.match_exact_fast(image, template, method, precision=precision, threads=3)
        assert np.array_equal(_bits(fast), _bits(plain))
        assert ext == O.find_extremes(plain)


def test_fast_extremes_first_occurrence_on_ties():
    # a periodic image makes every extreme a tie many times over
    image = np.tile(np.arange(8, dtype=np.uint8) * 30, (50, 12))
    template = image[:5, :9].copy()
    for method in range(4):
        plain = O.match_exact(image, template, method)
        for threads in (1, 4, 7):
            _, ext = O.match_exact_fast(image, template, method, threads=threads, want_map=False)
            assert ext == O.find_extremes(plain)


def test_many_fast_bands_and_extremes():
    rng = np.random.default_rng(5)
    image = rng.integers(0, 256, size=(90, 120), dtype=np.uint8)
    templates = rng.integers(0, 256, size=(5, 11, 20), dtype=np.uint8)
    maps, ext = O.many_exact_fast(image, templates, 3, rows=(7, 40), want_maps=True, threads=4)
    _, full_ext = O.many_exact_fast(image, templates, 3, threads=4)
    for k in range(5):
        plain = O.match_exact(image, templates[k], 3)
        assert np.array_equal(_bits(maps[k]), _bits(plain[7:40]))
        mx, mn, (mxx, mxy), (mnx, mny) = O.find_extremes(plain[7:40])
        assert ext[k] == (mx, mn, (mxx, mxy + 7), (mnx, mny + 7))
        assert full_ext[k] == O.find_extremes(plain)


def test_fast_rejects_templates_whose_sums_could_overflow():
    image = np.zeros((300, 300), np.uint8)
    with pytest.raises(O.OracleError):
        O.match_exact_fast(image, np.zeros((258, 258), np.uint8), 0)
