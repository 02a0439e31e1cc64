"""The row-operand tcgen05 kernel (image rows read in place as the A operand)
against the oracle.

Bar: bit-exact (same exact integer sums, same epilogue). Shapes cover every
K width the kernel takes (template widths + 15 rounded to 32, 64, 96, 128 and
160 bytes), maps narrower and wider than one 2048-column tile (two and three
tiles across, a map exactly one tile wide), partial 16-row tiles at the
bottom, one-row and one-column maps, templates of one pixel, zero norms and
sums near the 32-bit limit.
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


def run_rows(image, template, method, precision=tm.Precision.ExactFp64):
    tm.set_path(tm.Path.RowOperand)
    tm.set_precision(precision)
    _lib.profile_enable(True)
    _lib.profile_collect()
    got = tm.match_template(image, template, method)
    stats = _lib.profile_collect()
    _lib.profile_enable(False)
    assert stats.get("rows_i8", {}).get("launches", 0) >= 1, stats  # the row-operand kernel ran
    return got


SHAPES = [
    # (H, W), (h, w)
    ((300, 2112), (16, 16)),    # K = 32, two tiles across
    ((257, 512), (24, 40)),     # K = 64, one partial tile
    ((150, 4160), (33, 100)),   # K = 128, three tiles across
    ((200, 640), (64, 145)),    # K = 160, the widest template taken
    ((97, 272), (1, 1)),        # one-pixel template
    ((40, 256), (40, 17)),      # one output row
    ((50, 16), (9, 16)),        # one output column
    ((60, 160), (17, 145)),     # 16 output columns, K = 160
    ((130, 2064), (8, 17)),     # a map exactly one tile wide
    ((111, 1040), (48, 48)),    # K = 64 with 48-row template, partial bottom tile
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0][0]}x{s[0][1]}_t{s[1][0]}x{s[1][1]}")
def test_row_operand_bit_exact(shape):
    (H, W), (h, w) = shape
    g = np.random.default_rng(H * 13 + w)
    image = g.integers(0, 256, (H, W), dtype=np.uint8)
    template = g.integers(0, 256, (h, w), dtype=np.uint8)
    for method in M:
        got = run_rows(image, template, method)
        exp = O.match_exact(image, template, method, None, precision=0)
        bad = np.argwhere(bits(got) != bits(exp))
        assert bad.size == 0, (method, bad[:5], got[tuple(bad[0])], exp[tuple(bad[0])])


def test_row_operand_blob_scene_both_exact_precisions():
    image, template, _, _ = synthetic.blob_scene()
    for prec, code in ((tm.Precision.ExactFp64, 0), (tm.Precision.ExactF32, 1)):
        for method in M:
            got = run_rows(image, template, method, prec)
            exp = O.match_exact(image, template, method, None, precision=code)
            assert bits(got).tolist() == bits(exp).tolist(), (prec, method)


def test_row_operand_zero_norm_and_saturated_sums():
    # flat zero regions: Y = 0, the normalised methods fall back to the raw score
    image = np.zeros((120, 528), np.uint8)
    image[60:, 300:] = 255
    template = np.full((80, 100), 255, np.uint8)  # X and Y near 80 * 100 * 255^2 < 2^31
    for method in M:
        got = run_rows(image, template, method)
        exp = O.match_exact(image, template, method, None, precision=0)
        assert bits(got).tolist() == bits(exp).tolist(), method
    zero_t = np.zeros((20, 30), np.uint8)  # TSS = 0
    for method in M:
        got = run_rows(image, zero_t, method)
        exp = O.match_exact(image, zero_t, method, None, precision=0)
        assert bits(got).tolist() == bits(exp).tolist(), method


def test_row_operand_repeated_calls_and_fallback():
    g = np.random.default_rng(9)
    image = g.integers(0, 256, (90, 2100), dtype=np.uint8)  # width not a multiple of 16
    template = g.integers(0, 256, (10, 12), dtype=np.uint8)
    tm.set_path(tm.Path.RowOperand)
    got = tm.match_template(image, template, M.SumOfSquaredErrors)  # another kernel takes it
    assert bits(got).tolist() == bits(O.match_exact(image, template, M.SumOfSquaredErrors, None)).tolist()
    image = image[:, :2096].copy()
    first = run_rows(image, template, M.CrossCorrelationNormalized)
    for _ in range(3):
        again = run_rows(image, template, M.CrossCorrelationNormalized)
        assert bits(again).tolist() == bits(first).tolist()
    assert bits(first).tolist() == bits(O.match_exact(image, template, M.CrossCorrelationNormalized,
                                                       None)).tolist()


def _check_batch(items, outs, extremes):
    for k, ((image, template, method, mask), out, ex) in enumerate(zip(items, outs, extremes)):
        got = out.cpu().numpy()
        exp = O.match_exact(image, template, method, mask, precision=0)
        bad = np.argwhere(bits(got) != bits(exp))
        assert bad.size == 0, (k, image.shape, template.shape, method, mask is not None, bad[:3])
        mx, mn, mxl, mnl = O.find_extremes(exp)
        assert (ex.max_value, ex.min_value, ex.max_value_location, ex.min_value_location) == \
            (float(mx), float(mn), mxl, mnl), k


def _run_batch(items, replays=2):
    import torch

    from imageproc_b200 import device
    dev = []
    for image, template, method, mask in items:
        t = (torch.from_numpy(image).cuda(), torch.from_numpy(template).cuda(), method)
        dev.append(t if mask is None else t + (torch.from_numpy(mask).cuda(),))
    tm.set_path(tm.Path.RowOperand)
    batch = device.Batch(dev)
    batch.run()
    _check_batch(items, batch.outs, batch.extremes_host())
    plan = device.BatchPlan(batch)
    for _ in range(replays):
        for o in batch.outs:
            o.fill_(float("nan"))
        batch.extremes.zero_()
        plan.launch()
        torch.cuda.synchronize()
        _check_batch(items, batch.outs, batch.extremes_host())
    info = plan.info()
    plan.close()
    return info


def test_row_operand_batch_eight_map_step():
    # the benchmark's step: four unmasked maps (one row-operand launch, one
    # window-sum map for the three methods that need it) beside the four
    # binary-mask maps on the Hankel-row kernel
    image, template, mask, _ = synthetic.blob_scene()
    items = [(image, template, m, None) for m in M] + [(image, template, m, mask) for m in M]
    info = _run_batch(items)
    assert info["tensor_pairs"] == 8


def test_row_operand_batch_chunks_images_and_other_kernels():
    g = np.random.default_rng(17)
    imgs = [g.integers(0, 256, (200, 2112), dtype=np.uint8), g.integers(0, 256, (150, 640), dtype=np.uint8)]
    imgs[1][:40] = 9  # a flat band: ties for the extremes
    t1 = g.integers(0, 256, (20, 36), dtype=np.uint8)
    t2 = g.integers(0, 256, (11, 9), dtype=np.uint8)
    items = []
    for k in range(10):  # one template, two images, more pairs than one launch takes
        items.append((imgs[k % 2], t1, int(g.integers(0, 4)), None))
    for k in range(3):
        items.append((imgs[k % 2], t2, k, None))
    odd = g.integers(0, 256, (90, 301), dtype=np.uint8)  # width not a multiple of 16
    items.append((odd, t1, 3, None))
    items.append((imgs[0], t1, 0, (g.random(t1.shape) < 0.7).astype(np.uint8)))
    _run_batch(items, replays=1)
