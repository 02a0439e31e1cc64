"""Host-side checks of the rows beside the path (filter_clamped and its 1-D
forms, suppress_non_maximum / local_maxima, the integral images), without a
GPU: the errors the Python mirrors and the C ABI raise before any device work,
with the reference's panic messages where the reference panics, and the empty
inputs that need no device at all.
"""

import numpy as np
import pytest

from imageproc_b200 import filter as F
from imageproc_b200 import integral_image as II
from imageproc_b200 import suppress as S
from imageproc_b200._lib import Panic

IMG = np.zeros((4, 5), np.uint8)
K3 = np.ones((3, 3), np.float32)


def test_filter_zero_sized_kernel_panics_like_kernel_new():
    # Kernel::new (src/kernel.rs:24-33)
    for shape in ((0, 3), (3, 0)):
        with pytest.raises(Panic, match="^width and height must be non-zero$"):
            F.filter_clamped(IMG, np.zeros(shape, np.float32))


def test_separable_filter_kernels_of_different_lengths_panic():
    # separable_filter (src/filter/mod.rs:175-179)
    with pytest.raises(Panic, match="^the two 1D kernels must be the same length$"):
        F.separable_filter(IMG, np.ones(3, np.float32), np.ones(5, np.float32))


def test_filter_rejects_types_the_reference_has_no_instance_for():
    with pytest.raises(TypeError):
        F.filter_clamped(IMG.astype(np.uint16), K3)  # images are u8 Luma / Rgb / Rgba
    with pytest.raises(TypeError):
        F.filter_clamped(np.zeros((4, 5, 2), np.uint8), K3)
    with pytest.raises(TypeError):
        F.filter_clamped(IMG, K3.astype(np.float64))  # kernels are f32 or i32
    with pytest.raises(TypeError):
        F.filter_clamped(IMG, K3, np.float64)
    # an i32 kernel has no Clamp to f32: refused by the C ABI before any device work
    with pytest.raises(ValueError, match="no Clamp"):
        F.filter_clamped(IMG, np.ones((3, 3), np.int32), np.float32)


@pytest.mark.parametrize("shape", [(0, 5), (4, 0), (0, 0, 3)])
def test_filter_of_an_empty_image_is_empty(shape):
    out = F.filter_clamped(np.zeros(shape, np.uint8), K3)
    assert out.shape == shape and out.dtype == np.uint8


def test_suppress_rejects_unsupported_arrays():
    with pytest.raises(TypeError):
        S.suppress_non_maximum(np.zeros((4, 4), np.float64), 1)
    with pytest.raises(TypeError):
        S.suppress_non_maximum(np.zeros((4, 4, 3), np.uint8), 1)


def test_suppress_of_an_empty_image_is_empty():
    for shape in ((0, 7), (7, 0)):
        out = S.suppress_non_maximum(np.zeros(shape, np.float32), 2)
        assert out.shape == shape and out.dtype == np.float32


def test_local_maxima_of_no_points_keeps_none():
    assert S.local_maxima_indices([], [], [], 3) == []
    with pytest.raises(ValueError, match="one entry per point"):
        S.local_maxima_indices([1, 2], [1], [0.5, 0.5], 3)


def test_integral_images_reject_unsupported_arrays():
    with pytest.raises(TypeError):
        II.integral_image(IMG.astype(np.uint16))
    with pytest.raises(TypeError):
        II.integral_image(np.zeros((4, 5, 2), np.uint8))
    with pytest.raises(TypeError):
        II.integral_squared_image(IMG, dtype=np.uint16)
