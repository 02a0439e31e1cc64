"""Host-buffer match calls on large maps, which the library cuts into row
bands whose image copies, launches and score copies overlap. Every score must
still equal the oracle's bit for bit: a band is the window walk of
src/template_matching.rs:78-92 over a sub-range of output rows.

The cases cover odd widths (band starts that are not 16-byte aligned), the
tensor-core and CUDA-core families, binary and general masks, every
precision, and maps either side of the size where banding starts.
"""

import numpy as np
import pytest

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


def expected(image, template, method, mask, precision):
    if precision == P.ReferenceF32:
        return O.match_reference(image, template, method, mask)
    return O.match_exact(image, template, method, mask, precision=int(precision))


def scene(H, W, h, w, seed, mask_kind=None):
    g = np.random.default_rng(seed)
    image = g.integers(0, 256, (H, W), dtype=np.uint8)
    y, x = int(g.integers(0, H - h + 1)), int(g.integers(0, W - w + 1))
    template = image[y:y + h, x:x + w].copy()
    mask = None
    if mask_kind == "binary":
        mask = (g.random((h, w)) < 0.8).astype(np.uint8)
    elif mask_kind == "gray":
        mask = g.integers(0, 256, (h, w), dtype=np.uint8)
    return image, template, mask


# (H, W, h, w, mask): score maps of 1.9 to 8.8 MB
CASES = [
    (1080, 1920, 64, 64, None),      # the 1080p scene: 4 bands, tensor cores
    (2100, 1003, 9, 17, "binary"),   # odd width: unaligned band starts
    (1500, 1500, 20, 20, "gray"),    # general mask: CUDA-core family
    (700, 700, 16, 16, None),        # 1.85 MB: one band
    (745, 745, 16, 16, None),        # 2.04 MB: two bands
    (1100, 1601, 130, 7, None),      # tall template, thin: CUDA cores
]


@pytest.mark.parametrize("H,W,h,w,mask_kind", CASES)
def test_banded_host_calls_match_oracle(H, W, h, w, mask_kind):
    image, template, mask = scene(H, W, h, w, H + W, mask_kind)
    for k, method in enumerate(M):
        precision = (P.ExactFp64, P.ExactF32, P.ReferenceF32, P.ExactFp64)[k]
        if precision == P.ReferenceF32 and H * W * h * w > 2e9:
            precision = P.ExactF32  # keep the oracle's f32 walk short
        tm.set_precision(precision)
        got = (tm.match_template(image, template, method) if mask is None
               else tm.match_template_with_mask(image, template, method, mask))
        exp = expected(image, template, method, mask, precision)
        assert got.shape == exp.shape
        assert np.array_equal(bits(got), bits(exp)), (method, precision)


def test_banded_calls_repeat_and_interleave_sizes():
    """A large call, a small one and a large one again on the same thread
    reuse the context's buffers and copy streams; each must be exact."""
    tm.set_precision(P.ExactFp64)
    big = scene(1080, 1920, 32, 48, 1)
    small = scene(100, 120, 16, 16, 2)
    other = scene(1200, 1777, 24, 40, 3, "binary")
    for image, template, mask in (big, small, other, big):
        for method in (M.SumOfSquaredErrors, M.CrossCorrelationNormalized):
            got = (tm.match_template(image, template, method) if mask is None
                   else tm.match_template_with_mask(image, template, method, mask))
            assert np.array_equal(bits(got), bits(expected(image, template, method, mask, P.ExactFp64)))
