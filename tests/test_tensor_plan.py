"""The tensor-core tile planner, on the host, for every template shape the
tensor path takes (ipb_tensor_plan_for: host arithmetic, no device work).

What every plan must hold, because the kernel relies on it without checking:
  * dynamic shared memory within the 227 KB a CTA may have, and at least
    120 KB, so that one CTA fits an SM: the launches of a batch plan run side
    by side and must never share an SM's tensor memory;
  * accumulators plus A stages within the 512 tensor-memory columns;
  * a tile's image rows within the 256-entry band table, including the MMA
    loop's read-ahead of up to three entries past the last row;
  * s32 accumulation exact: every window sum below 2^31;
  * a batch group's plan wherever a single launch has one (a pair the
    library sends to the tensor path must find a plan in its group).
"""

import pytest

from imageproc_b200 import _lib

SMEM_MAX = 227 * 1024
SMEM_ONE_CTA_PER_SM = 120 * 1024
TMEM_COLUMNS = 512
BAND_TABLE_ROWS = 256
BAND_TABLE_OFFSET = 1024


def shape_taken(w, h, masked):
    return w >= 8 and 8 <= h <= 128 and w <= (128 if masked else 256) and w * h <= 33025


def shapes():
    for masked in (False, True):
        for h in range(8, 129):
            for w in range(8, 257):
                if shape_taken(w, h, masked):
                    yield w, h, masked


@pytest.mark.parametrize("masked", [False, True])
def test_every_taken_shape_has_a_plan_within_the_hardware(masked):
    checked = 0
    for w, h, m in shapes():
        if m != masked:
            continue
        single = _lib.tensor_plan(w, h, m, batch=False)
        group = _lib.tensor_plan(w, h, m, batch=True)
        if single is None:
            continue  # the shape runs on CUDA cores
        assert group is not None, (w, h, m)
        for p in (single, group):
            assert SMEM_ONE_CTA_PER_SM <= p["smem_bytes"] <= SMEM_MAX, (w, h, m, p)
            assert p["tmem_columns"] <= TMEM_COLUMNS, (w, h, m, p)
            assert p["image_rows"] == p["tile_rows"] + h - 1
            assert p["image_rows"] <= BAND_TABLE_ROWS, (w, h, m, p)
            assert BAND_TABLE_OFFSET + (p["image_rows"] + 3) * 16 <= p["smem_bytes"]
            assert 1 <= p["rows_per_stage"] <= 16 and p["stages"] == 2
            assert p["image_buffers"] in (1, 2)
            assert p["tile_rows"] % 16 == 0
        checked += 1
    assert checked > 10000


def test_window_sums_fit_s32_for_every_taken_shape():
    for w, h, masked in shapes():
        if _lib.tensor_plan(w, h, masked, batch=False) is None:
            continue
        # X = sum I*T(*m) and, masked, Y = sum I^2*m: both at most 255^2 per pixel
        assert 255 * 255 * w * h < 2 ** 31, (w, h, masked)


def test_shapes_outside_the_tensor_path_have_no_plan():
    for w, h, masked in [(7, 8, False), (7, 16, True), (16, 7, False), (16, 129, False), (257, 8, False),
                         (129, 8, True), (256, 130, False)]:
        assert _lib.tensor_plan(w, h, masked, batch=False) is None


def test_plans_of_the_headline_shapes():
    # 64x64 templates of the 1080p scene: unmasked tiles of 128 rows with 12
    # rows per stage; binary-mask tiles of 96 rows in batch plans (3 rows per
    # stage) and of 64 rows in single launches (4 rows per stage)
    u = _lib.tensor_plan(64, 64, False, batch=True)
    assert (u["tile_rows"], u["rows_per_stage"], u["image_buffers"]) == (128, 12, 2)
    assert _lib.tensor_plan(64, 64, False, batch=False) == u
    mb = _lib.tensor_plan(64, 64, True, batch=True)
    assert (mb["tile_rows"], mb["rows_per_stage"], mb["image_buffers"]) == (96, 3, 2)
    ms = _lib.tensor_plan(64, 64, True, batch=False)
    assert (ms["tile_rows"], ms["rows_per_stage"], ms["image_buffers"]) == (64, 4, 2)


@pytest.mark.parametrize("masked", [False, True])
def test_set_plans_within_the_hardware(masked):
    # pairs on one image are computed in sets of 2..4: every member's
    # accumulators and template side must fit beside the A stages, and the
    # kernel's shared-memory header (TSS partials and keys per member slot)
    # stays below the band table. Where no set plan fits, the planner
    # computes the pairs alone, which the single-pair plan above covers.
    planned = 0
    for w, h, m in shapes():
        if m != masked or _lib.tensor_plan(w, h, m, batch=True) is None:
            continue
        for n in (1, 2, 3, 4):
            p = _lib.tensor_set_plan(w, h, m, n)
            if n == 1:
                assert p is not None, (w, h, m)
            if p is None:
                continue
            planned += 1
            assert SMEM_ONE_CTA_PER_SM <= p["smem_bytes"] <= SMEM_MAX, (w, h, m, n, p)
            assert p["tmem_columns"] <= TMEM_COLUMNS, (w, h, m, n, p)
            assert p["image_rows"] == p["tile_rows"] + h - 1 <= BAND_TABLE_ROWS
            assert BAND_TABLE_OFFSET + (p["image_rows"] + 3) * 16 <= p["smem_bytes"]
            assert 1 <= p["rows_per_stage"] <= 16 and p["tile_rows"] % 16 == 0
    assert planned > 20000


def test_set_plans_of_the_headline_shapes():
    # 64x64 templates: four unmasked maps per set on 64-row tiles (the four
    # accumulators take 256 columns, 8 image rows per stage); four
    # binary-mask maps per set on 64-row tiles (four X accumulators and the
    # set's common Y, 2 image rows of 3 planes per stage)
    p = _lib.tensor_set_plan(64, 64, False, 4)
    assert (p["tile_rows"], p["rows_per_stage"], p["tmem_columns"]) == (64, 8, 4 * 64 + 2 * 16 * 8)
    p = _lib.tensor_set_plan(64, 64, True, 4)
    assert (p["tile_rows"], p["rows_per_stage"], p["tmem_columns"]) == (64, 2, 5 * 64 + 2 * 3 * 16 * 2)
    assert _lib.tensor_set_plan(64, 64, False, 5) is None
