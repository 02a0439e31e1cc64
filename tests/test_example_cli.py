"""The host half of the example workflow (examples/template_matching.rs): image
files, argument handling and the oracle's rescale / outline, on the CPU."""

import struct
import zlib

import numpy as np
import pytest

from imageproc_b200 import png
from imageproc_b200._lib import Panic
from imageproc_b200.examples import template_matching as ex
from oracle import oracle as O


def _filtered_png(img: np.ndarray, ftypes) -> bytes:
    """A PNG whose rows use the given filter types (PNG spec filter definitions)."""
    a = np.asarray(img, np.uint8)
    h, w = a.shape[:2]
    ch = 1 if a.ndim == 2 else a.shape[2]
    rows = a.reshape(h, w * ch).astype(np.int32)
    raw = bytearray()
    prior = np.zeros(w * ch, np.int32)
    for y in range(h):
        ft = ftypes[y % len(ftypes)]
        cur = rows[y]
        left = np.concatenate([np.zeros(ch, np.int32), cur[:-ch]])
        upleft = np.concatenate([np.zeros(ch, np.int32), prior[:-ch]])
        if ft == 0:
            f = cur
        elif ft == 1:
            f = cur - left
        elif ft == 2:
            f = cur - prior
        elif ft == 3:
            f = cur - (left + prior) // 2
        else:
            p = left + prior - upleft
            pa, pb, pc = np.abs(p - left), np.abs(p - prior), np.abs(p - upleft)
            pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prior, upleft))
            f = cur - pred
        raw += bytes([ft]) + (f & 0xFF).astype(np.uint8).tobytes()
        prior = cur
    ctype = {1: 0, 2: 4, 3: 2, 4: 6}[ch]

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0))
            + chunk(b"IDAT", zlib.compress(bytes(raw))) + chunk(b"IEND", b""))


@pytest.mark.parametrize("channels", [1, 2, 3, 4])
def test_png_decodes_every_filter(channels):
    g = np.random.default_rng(channels)
    img = g.integers(0, 256, (23, 17) if channels == 1 else (23, 17, channels), dtype=np.uint8)
    got = png.decode_png(_filtered_png(img, [0, 1, 2, 3, 4]))
    assert np.array_equal(got, img)


def test_png_and_netpbm_round_trips(tmp_path):
    g = np.random.default_rng(0)
    gray = g.integers(0, 256, (31, 45), dtype=np.uint8)
    rgb = g.integers(0, 256, (12, 9, 3), dtype=np.uint8)
    for img in (gray, rgb):
        png.write_png(tmp_path / "a.png", img)
        assert np.array_equal(png.read_image(tmp_path / "a.png"), img)
    (tmp_path / "a.pgm").write_bytes(b"P5\n# comment\n45 31\n255\n" + gray.tobytes())
    assert np.array_equal(png.read_image(tmp_path / "a.pgm"), gray)
    (tmp_path / "a.ppm").write_bytes(b"P6 9 12 255\n" + rgb.tobytes())
    assert np.array_equal(png.read_image(tmp_path / "a.ppm"), rgb)


def test_to_luma8():
    rgb = np.array([[[255, 255, 255], [255, 0, 0], [0, 255, 0], [0, 0, 255], [10, 20, 30]]], np.uint8)
    want = [(2126 * r + 7152 * g_ + 722 * b) // 10000 for r, g_, b in rgb[0].astype(int)]
    assert png.to_luma8(rgb)[0].tolist() == want
    rgba = np.concatenate([rgb, np.full((1, 5, 1), 7, np.uint8)], axis=2)
    assert np.array_equal(png.to_luma8(rgba), png.to_luma8(rgb))
    la = np.stack([np.arange(5, dtype=np.uint8), np.full(5, 9, np.uint8)], axis=1)[None]
    assert png.to_luma8(la)[0].tolist() == [0, 1, 2, 3, 4]


def test_arguments_and_panics(tmp_path):
    with pytest.raises(Panic, match="Usage"):
        ex.parse_args(["prog", "in.png", "out", "1", "2", "3"])
    with pytest.raises(Panic, match="ParseIntError"):
        ex.parse_args(["prog", "in.png", "out", "1", "-2", "3", "4"])
    with pytest.raises(Panic, match="ParseBoolError"):
        ex.parse_args(["prog", "in.png", "out", "1", "2", "3", "4", "yes"])
    a = ex.parse_args(["prog", "in.png", "out", "+1", "2", "3", "4", "true"])
    assert (a["template_x"], a["template_h"], a["parallel"]) == (1, 4, True)
    with pytest.raises(Panic, match="^Input file does not exist$"):
        ex.main(["prog", str(tmp_path / "missing.png"), str(tmp_path / "out"), "1", "2", "3", "4"])
    assert (tmp_path / "out").is_dir()  # created before the input check, as the reference does
    with pytest.raises(Panic, match="Failed to create output directory"):
        ex.main(["prog", "x.png", str(tmp_path / "no" / "such"), "1", "2", "3", "4"])


def test_oracle_rescale_and_outline():
    s = np.array([[0, 1, 2], [3, np.nan, 4]], np.float32)
    assert O.convert_to_gray_image(s).tolist() == [[0, 63, 127], [191, 0, 255]]
    assert not O.convert_to_gray_image(np.full((2, 2), 5, np.float32)).any()  # range 0: NaN -> 0
    rgb = O.draw_green_rect(np.full((5, 6), 9, np.uint8), 4, 3, 4, 4)  # clipped at the right and bottom
    green = (rgb == [0, 255, 0]).all(axis=2)
    want = np.zeros((5, 6), bool)
    want[3, 4:] = want[3:, 4] = True
    assert np.array_equal(green, want)
    assert (rgb[~green] == 9).all()
    with pytest.raises(AssertionError, match="invalid sub-image"):
        O.template_matching_example(np.zeros((10, 10), np.uint8), 5, 0, 5, 3)
