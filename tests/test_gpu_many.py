"""Many templates against one image (ipb_match_templates_device) against the oracle.

Bar: every template's score map bit-exact against the oracle's exact-sum
epilogue; per-template extremes equal to the oracle's find_extremes
(src/template_matching.rs:479-511) of that map.
"""

import numpy as np
import pytest

from imageproc_b200 import synthetic
from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu
M = tm.MatchTemplateMethod


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _run(image, templates, method, precision=tm.Precision.ExactFp64, extremes=True):
    import torch

    from imageproc_b200 import device
    di = torch.from_numpy(image).cuda()
    dt = torch.from_numpy(templates).cuda()
    out, ex = device.match_templates_device(di, dt, method, precision=precision, extremes=extremes)
    torch.cuda.synchronize()
    return out.cpu().numpy(), ex


CASES = [
    # (H, W), (n, h, w)
    # positions as the MMA's M side (banks of at most 64, or large templates)
    ((300, 512), (40, 32, 32)),    # aligned image rows, n not a multiple of the block
    ((257, 333), (21, 24, 16)),    # odd sizes, n % 4 != 0 (scalar score stores)
    ((200, 260), (18, 48, 48)),    # smaller template blocks
    ((190, 300), (33, 64, 64)),
    ((170, 200), (90, 40, 40)),    # a bank of 90 that does not fit as 128 templates
    # templates as the MMA's M side (blocks of 128)
    ((140, 150), (130, 8, 20)),    # two blocks, the second with 2 templates
    ((260, 300), (100, 32, 32)),   # one partial block
    ((190, 333), (70, 16, 16)),    # odd image width (no cp.async staging)
    ((150, 200), (129, 36, 32)),   # the tallest template whose block fits
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0][0]}x{c[0][1]}_n{c[1][0]}_{c[1][1]}x{c[1][2]}")
def test_many_templates_bit_exact(case):
    (H, W), (n, h, w) = case
    g = np.random.default_rng(H + 13 * n)
    image = g.integers(0, 256, (H, W), dtype=np.uint8)
    templates = g.integers(0, 256, (n, h, w), dtype=np.uint8)
    templates[0] = image[5:5 + h, 7:7 + w]  # one exact crop: a unique best match
    for method in (M.CrossCorrelationNormalized, M.SumOfSquaredErrors):
        out, ex = _run(image, templates, method)
        assert out.shape == (H - h + 1, W - w + 1, n)
        for t in range(n):
            exp = O.match_exact(image, templates[t], method, None, precision=0)
            bad = np.argwhere(bits(out[:, :, t]) != bits(exp))
            assert bad.size == 0, (t, method, bad[:3])
            mx, mn, mxl, mnl = O.find_extremes(exp)
            e = ex[t]
            assert (e.max_value, e.min_value, e.max_value_location, e.min_value_location) == \
                (float(mx), float(mn), mxl, mnl), (t, method)


@pytest.mark.parametrize("n", [20, 100])  # positions as M, templates as M
def test_many_templates_extremes_ties_first_occurrence(n):
    # a periodic scene: every template's best (and worst) score repeats every
    # 16 pixels, so the record must name the first occurrence in row-major order
    g = np.random.default_rng(5)
    tile = g.integers(0, 256, (16, 16), dtype=np.uint8)
    image = np.tile(tile, (14, 20))
    templates = np.stack([image[(t % 7):(t % 7) + 32, (t % 5):(t % 5) + 32] for t in range(n)])
    for method in M:
        out, ex = _run(image, templates, method)
        for t in range(0, n, 7):
            exp = O.match_exact(image, templates[t], method, None, precision=0)
            assert bits(out[:, :, t]).tolist() == bits(exp).tolist()
            mx, mn, mxl, mnl = O.find_extremes(exp)
            e = ex[t]
            assert (e.max_value, e.min_value, e.max_value_location, e.min_value_location) == \
                (float(mx), float(mn), mxl, mnl), (t, method)
    # an all-zero scene: every score ties (zero norm keeps the raw score, 0)
    zero = np.zeros((120, 150), np.uint8)
    out, ex = _run(zero, templates, M.CrossCorrelationNormalized)
    assert not out.any()
    assert all(e.max_value_location == (0, 0) and e.min_value_location == (0, 0) for e in ex)


def test_many_templates_all_methods_and_f32_precision():
    g = np.random.default_rng(9)
    image = g.integers(0, 256, (180, 300), dtype=np.uint8)
    templates = g.integers(0, 256, (12, 32, 32), dtype=np.uint8)
    for method in M:
        for prec in (tm.Precision.ExactFp64, tm.Precision.ExactF32):
            out, _ = _run(image, templates, method, prec, extremes=False)
            for t in range(12):
                exp = O.match_exact(image, templates[t], method, None, precision=int(prec))
                assert bits(out[:, :, t]).tolist() == bits(exp).tolist()


@pytest.mark.parametrize("n", [48, 160])
def test_value_noise_workload_reduced(n):
    # the many-templates workload's generator at a reduced size
    image, templates, locs = synthetic.value_noise_scene(W=512, H=384, n_templates=n, t=32, seed=4)
    out, ex = _run(image, templates, M.CrossCorrelationNormalized)
    for t in range(0, n, 5):
        exp = O.match_exact(image, templates[t], M.CrossCorrelationNormalized, None, precision=0)
        assert bits(out[:, :, t]).tolist() == bits(exp).tolist()
        mx, mn, mxl, mnl = O.find_extremes(exp)
        assert (ex[t].max_value, ex[t].max_value_location) == (float(mx), mxl)


def test_many_templates_rejects_unsupported_shapes():
    import torch

    from imageproc_b200 import device
    img = torch.zeros((100, 100), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        device.match_templates_device(img, torch.zeros((3, 8, 8), dtype=torch.uint8, device="cuda"), 0)
    with pytest.raises(tm.Panic, match="^image width must be greater than or equal to template width$"):
        device.match_templates_device(img, torch.zeros((3, 8, 101), dtype=torch.uint8, device="cuda"), 0)
