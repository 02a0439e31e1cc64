"""The allocation-free entry point, checked against the oracle and the ordinary device entry point.

ipb_match_template_device_noalloc serves callers that cannot call cudaMalloc
(a plug-in inside an application that owns the device-memory budget, or a loop
where an allocation would stall the device): its scratch memory is a fixed
array inside the library. This file is collected last so that a failure here
never hides the result of another test; it passes alone in a fresh process and
after the rest of the suite.
"""

import numpy as np
import pytest

from imageproc_b200 import _lib, synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EXACT_FP64, EXACT_F32, REFERENCE_F32 = 0, 1, 2
SCRATCH_LIMIT = 16 << 20  # the entry point's fixed scratch array


def _call(fn, image, template, mask, binary, method, precision, out, stream):
    H, W = image.shape
    h, w = template.shape
    mh, mw = mask.shape if mask is not None else (0, 0)
    return fn(image.data_ptr(), W, H, template.data_ptr(), w, h,
              mask.data_ptr() if mask is not None else None, mw, mh,
              int(binary), method, precision, out.data_ptr(), stream)


def _oracle(image, template, method, mask, precision):
    if precision == REFERENCE_F32:
        return O.match_reference(image, template, method, mask)
    return O.match_exact(image, template, method, mask, precision=precision)


def _general_mask(shape, seed):
    # arbitrary u8 weights, as the reference's masks are (its own test uses 0..3)
    return np.random.default_rng(seed).integers(0, 256, size=shape, dtype=np.uint8)


def test_noalloc_matches_oracle_and_device_entry_point_twice_in_a_row():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream or None
    # different problems back to back: a call must not see the previous call's
    # leftovers in the shared scratch array
    img1, tpl1, mask1, _ = synthetic.blob_scene(W=1920, H=1080, tw=64, th=64, seed=31)
    img2, tpl2, mask2, _ = synthetic.blob_scene(W=700, H=500, tw=40, th=24, seed=32)
    gmask2 = _general_mask(tpl2.shape, 33)
    cases = [
        (img1, tpl1, None, False, 1, EXACT_FP64),    # SSE-normalised: uses the integral image
        (img2, tpl2, mask2, True, 3, EXACT_FP64),    # binary-mask CCORR-normalised
        (img2, tpl2, gmask2, False, 1, EXACT_FP64),  # general u8 mask, SSE-normalised
        (img2, tpl2, gmask2, False, 2, EXACT_F32),   # general u8 mask, CCORR
        (img2, tpl2, None, False, 3, EXACT_F32),     # reference f32 normalisation of exact sums
        (img1, tpl1, mask1, True, 0, EXACT_F32),
        (img2, tpl2, None, False, 0, REFERENCE_F32),
    ]
    for image, template, mask, binary, method, precision in cases:
        exp = _oracle(image, template, method, mask, precision).view(np.uint32)
        di = torch.from_numpy(image).to(dev)
        dt = torch.from_numpy(template).to(dev)
        dm = torch.from_numpy(mask).to(dev) if mask is not None else None
        shape = exp.shape
        ref = torch.empty(shape, dtype=torch.float32, device=dev)
        _lib.check(_call(L.ipb_match_template_device, di, dt, dm, binary, method, precision, ref,
                         stream))
        torch.cuda.synchronize()
        assert np.array_equal(ref.cpu().numpy().view(np.uint32), exp)
        for _ in range(2):
            got = torch.full(shape, float("nan"), dtype=torch.float32, device=dev)
            _lib.check(_call(L.ipb_match_template_device_noalloc, di, dt, dm, binary, method,
                             precision, got, stream))
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy().view(np.uint32), exp), \
                (method, precision, mask is not None, binary)


def _scratch_need_unmasked_sse(W, H, w, h):
    # template plane (rows padded to 64 bytes) + the template constant, then the
    # u64 integral image of I^2, each rounded up to 256 bytes
    planes = -(-(h * -(-w // 64) * 64) // 256) * 256 + 256
    return planes + -(-((W + 1) * (H + 1) * 8) // 256) * 256


def test_noalloc_scratch_limit_is_exact():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    # (W+1)(H+1) * 8 + 1280 == 16 MiB exactly for a 3448 x 607 image and a 16 x 16 template
    W, H, w, h = 3448, 607, 16, 16
    assert _scratch_need_unmasked_sse(W, H, w, h) == SCRATCH_LIMIT
    assert _scratch_need_unmasked_sse(W, H + 1, w, h) > SCRATCH_LIMIT
    rng = np.random.default_rng(41)
    image = rng.integers(0, 256, size=(H + 1, W), dtype=np.uint8)
    template = image[100:100 + h, 200:200 + w].copy()
    dt = torch.from_numpy(template).to(dev)

    # exactly at the limit: accepted, and exact
    fits = image[:H]
    di = torch.from_numpy(np.ascontiguousarray(fits)).to(dev)
    out = torch.empty((H - h + 1, W - w + 1), dtype=torch.float32, device=dev)
    _lib.check(_call(L.ipb_match_template_device_noalloc, di, dt, None, False, 0, EXACT_FP64, out,
                     None))
    torch.cuda.synchronize()
    exp = O.match_exact(fits, template, 0, None, precision=EXACT_FP64)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), exp.view(np.uint32))

    # one image row more: rejected before any device work, with the sizes named
    di = torch.from_numpy(image).to(dev)
    out = torch.empty((H + 1 - h + 1, W - w + 1), dtype=torch.float32, device=dev)
    st = _call(L.ipb_match_template_device_noalloc, di, dt, None, False, 0, EXACT_FP64, out, None)
    assert st == _lib.ERR_INVALID_ARGUMENT
    msg = L.ipb_last_error_message().decode()
    assert "fixed maximum" in msg and str(SCRATCH_LIMIT) in msg


def test_noalloc_rejects_problems_above_its_fixed_scratch():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    image = torch.zeros((3000, 3000), dtype=torch.uint8, device=dev)  # 72 MB integral image
    template = torch.zeros((16, 16), dtype=torch.uint8, device=dev)
    out = torch.empty((2985, 2985), dtype=torch.float32, device=dev)
    st = _call(L.ipb_match_template_device_noalloc, image, template, None, False, 0, EXACT_FP64,
               out, None)
    assert st == _lib.ERR_INVALID_ARGUMENT
    msg = L.ipb_last_error_message().decode()
    assert "fixed maximum" in msg and "bytes" in msg
