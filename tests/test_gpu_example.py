"""The example workflow of examples/template_matching.rs as one device pipeline
(ipb_example_template_matching) against the oracle's restatement: template,
outlined image and both outlined, rescaled, padded score maps, byte for byte,
at each precision; then the command line end to end through PNG files."""

import numpy as np
import pytest

from imageproc_b200 import png, synthetic
from imageproc_b200 import template_matching as tm
from imageproc_b200._lib import Panic
from imageproc_b200.examples import template_matching as ex
from oracle import oracle as O

pytestmark = pytest.mark.gpu
NAMES = ("template", "image", "result_sse", "result_sse_norm")


@pytest.fixture(autouse=True)
def _restore_precision():
    old = tm.get_precision()
    yield
    tm.set_precision(old)


@pytest.mark.parametrize("precision", [tm.Precision.ExactFp64, tm.Precision.ExactF32, tm.Precision.ReferenceF32])
def test_pipeline_matches_oracle(precision):
    img, _, _, _ = synthetic.blob_scene()
    img = np.ascontiguousarray(img[:360, :500])
    tm.set_precision(precision)
    for x, y, w, h in ((100, 60, 48, 32), (0, 0, 17, 9), (440, 300, 59, 59), (3, 200, 1, 1)):
        got = ex.run_pipeline(img, x, y, w, h)
        exp = O.template_matching_example(img, x, y, w, h, precision=int(precision))
        for k in NAMES:
            assert got[k].shape == exp[k].shape, k
            assert np.array_equal(got[k], exp[k]), (k, x, y, w, h)


def test_pipeline_full_scene_and_odd_sizes():
    tm.set_precision(tm.Precision.ExactFp64)
    img, _, _, _ = synthetic.blob_scene()
    got = ex.run_pipeline(img, 900, 500, 64, 64)
    exp = O.template_matching_example(img, 900, 500, 64, 64)
    for k in NAMES:
        assert np.array_equal(got[k], exp[k]), k
    g = np.random.default_rng(7)
    odd = g.integers(0, 256, (101, 257), dtype=np.uint8)  # rows not a multiple of 4 pixels
    for k, v in ex.run_pipeline(odd, 5, 7, 33, 20).items():
        assert np.array_equal(v, O.template_matching_example(odd, 5, 7, 33, 20)[k]), k


def test_pipeline_assertion():
    img = np.zeros((50, 60), np.uint8)
    with pytest.raises(Panic, match="^invalid sub-image$"):
        ex.run_pipeline(img, 10, 10, 50, 5)  # x + w == width
    with pytest.raises(Panic, match="^invalid sub-image$"):
        ex.run_pipeline(img, 0, 45, 5, 5)


@pytest.mark.parametrize("rgb_input", [False, True])
def test_command_line_end_to_end(tmp_path, rgb_input):
    tm.set_precision(tm.Precision.ExactFp64)
    g = np.random.default_rng(3)
    if rgb_input:
        src = g.integers(0, 256, (140, 190, 3), dtype=np.uint8)
    else:
        src, _, _, _ = synthetic.blob_scene()
        src = np.ascontiguousarray(src[:150, :210])
    png.write_png(tmp_path / "in.png", src)
    ex.main(["prog", str(tmp_path / "in.png"), str(tmp_path / "out"), "30", "40", "25", "20", "true"])
    exp = O.template_matching_example(png.to_luma8(src), 30, 40, 25, 20)
    files = {"template": "template.png", "image": "image.png", "result_sse": "result_sse.png",
             "result_sse_norm": "result_sse_norm.png"}
    for k, f in files.items():
        assert np.array_equal(png.read_image(tmp_path / "out" / f), exp[k]), f
