"""The tcgen05 kind::i8 tensor-core path against the oracle and the CUDA-core path.

Bar: bit-exact (same exact integer sums, same epilogue). Shapes cover every
tensor-memory row width the kernel instantiates (template widths rounded to
32/64/128/256 bytes), both tile heights (128 and 64 output rows), image widths
that are and are not multiples of 16 bytes, and partial tiles at every edge.
"""

import numpy as np
import pytest

from imageproc_b200 import _lib, synthetic
from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu
M = tm.MatchTemplateMethod


@pytest.fixture(autouse=True)
def _restore():
    old_p, old_path = tm.get_precision(), tm.get_path()
    yield
    tm.set_precision(old_p)
    tm.set_path(old_path)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def run(image, template, method, path, precision=tm.Precision.ExactFp64):
    tm.set_path(path)
    tm.set_precision(precision)
    return tm.match_template(image, template, method)


SHAPES = [
    # (H, W), (h, w)
    ((300, 400), (16, 16)),     # 32-byte rows
    ((257, 333), (24, 40)),     # 64-byte rows, odd widths
    ((200, 512), (64, 64)),     # aligned width: 16-byte staging loads
    ((150, 700), (33, 100)),    # 128-byte rows
    ((180, 900), (128, 100)),   # tall template
    ((400, 600), (100, 256)),   # 256-byte rows, 64-row tiles
    ((130, 130), (8, 17)),      # short template
    ((64, 300), (64, 20)),      # one output row band
    ((150, 333), (12, 9)),      # narrow template: half of the first K step
    ((97, 260), (8, 8)),        # the narrowest and shortest template taken
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0][0]}x{s[0][1]}_t{s[1][0]}x{s[1][1]}")
def test_tensor_path_bit_exact(shape):
    (H, W), (h, w) = shape
    g = np.random.default_rng(H * 7 + w)
    image = g.integers(0, 256, (H, W), dtype=np.uint8)
    template = g.integers(0, 256, (h, w), dtype=np.uint8)
    launches0 = _lib.launch_count()
    for method in M:
        got = run(image, template, method, tm.Path.TensorCores)
        exp = O.match_exact(image, template, method, None, precision=0)
        bad = np.argwhere(bits(got) != bits(exp))
        assert bad.size == 0, (method, bad[:5], got[tuple(bad[0])], exp[tuple(bad[0])])
    assert _lib.launch_count() > launches0


def test_tensor_and_cuda_core_paths_agree_on_saturated_input():
    image = np.full((300, 520), 255, np.uint8)
    image[::3, ::7] = 0
    template = np.full((128, 256), 255, np.uint8)  # sums near the s32 limit
    for method in M:
        a = run(image, template, method, tm.Path.TensorCores)
        b = run(image, template, method, tm.Path.CudaCores)
        assert bits(a).tolist() == bits(b).tolist()


def test_tensor_path_blob_scene_all_methods_exact_f32():
    image, template, _, _ = synthetic.blob_scene()
    for method in M:
        got = run(image, template, method, tm.Path.TensorCores, tm.Precision.ExactF32)
        exp = O.match_exact(image, template, method, None, precision=1)
        assert bits(got).tolist() == bits(exp).tolist()


MASK_SHAPES = [s for s in SHAPES if s[1][1] <= 128]


@pytest.mark.parametrize("shape", MASK_SHAPES, ids=lambda s: f"{s[0][0]}x{s[0][1]}_t{s[1][0]}x{s[1][1]}")
def test_tensor_path_binary_mask_bit_exact(shape):
    (H, W), (h, w) = shape
    g = np.random.default_rng(H * 11 + w)
    image = g.integers(0, 256, (H, W), dtype=np.uint8)
    template = g.integers(0, 256, (h, w), dtype=np.uint8)
    mask = (g.random((h, w)) < 0.8).astype(np.uint8)
    tm.set_path(tm.Path.TensorCores)
    tm.set_precision(tm.Precision.ExactFp64)
    for method in M:
        got = tm.match_template_with_mask(image, template, method, mask)
        exp = O.match_exact(image, template, method, mask, precision=0)
        bad = np.argwhere(bits(got) != bits(exp))
        assert bad.size == 0, (method, bad[:5], got[tuple(bad[0])], exp[tuple(bad[0])])


def test_tensor_path_binary_mask_extremes():
    g = np.random.default_rng(5)
    image = g.integers(0, 256, (200, 300), dtype=np.uint8)
    template = g.integers(0, 256, (40, 48), dtype=np.uint8)
    tm.set_path(tm.Path.TensorCores)
    for mask in (np.zeros((40, 48), np.uint8), np.ones((40, 48), np.uint8)):
        for method in M:
            got = tm.match_template_with_mask(image, template, method, mask)
            exp = O.match_exact(image, template, method, mask, precision=0)
            assert bits(got).tolist() == bits(exp).tolist()
    ones = np.ones((40, 48), np.uint8)
    for method in M:
        a = tm.match_template_with_mask(image, template, method, ones)
        b = tm.match_template(image, template, method)
        assert bits(a).tolist() == bits(b).tolist()
