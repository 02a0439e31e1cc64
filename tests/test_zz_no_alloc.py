"""The allocation-free entry point, checked against the ordinary device entry point.

ipb_match_template_device_noalloc serves callers that cannot call cudaMalloc
(a plug-in inside an application that owns the device-memory budget, or a loop
where an allocation would stall the device): its scratch memory is a fixed
array inside the library. This file is collected last so that a failure here
never hides the result of another test; it passes alone in a fresh process and
after the rest of the suite.
"""

import ctypes as C

import numpy as np
import pytest

from imageproc_b200 import _lib, synthetic

pytestmark = pytest.mark.gpu

EXACT_FP64, REFERENCE_F32 = 0, 2


def _call(fn, image, template, mask, method, precision, out, stream):
    H, W = image.shape
    h, w = template.shape
    mh, mw = mask.shape if mask is not None else (0, 0)
    return fn(image.data_ptr(), W, H, template.data_ptr(), w, h,
              mask.data_ptr() if mask is not None else None, mw, mh,
              int(mask is not None), method, precision, out.data_ptr(), stream)


def test_noalloc_matches_device_entry_point_twice_in_a_row():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream or None
    # two different problems back to back: the second call must not see the
    # first call's leftovers in the shared scratch array
    img1, tpl1, mask1, _ = synthetic.blob_scene(W=1920, H=1080, tw=64, th=64, seed=31)
    img2, tpl2, mask2, _ = synthetic.blob_scene(W=700, H=500, tw=40, th=24, seed=32)
    cases = [
        (img1, tpl1, None, 1, EXACT_FP64),   # SSE-normalised: uses the integral image
        (img2, tpl2, mask2, 3, EXACT_FP64),  # masked CCORR-normalised
        (img2, tpl2, None, 0, REFERENCE_F32),
    ]
    for image, template, mask, method, precision in cases:
        di = torch.from_numpy(image).to(dev)
        dt = torch.from_numpy(template).to(dev)
        dm = torch.from_numpy(mask).to(dev) if mask is not None else None
        shape = (image.shape[0] - template.shape[0] + 1, image.shape[1] - template.shape[1] + 1)
        ref = torch.empty(shape, dtype=torch.float32, device=dev)
        _lib.check(_call(L.ipb_match_template_device, di, dt, dm, method, precision, ref, stream))
        for _ in range(2):
            got = torch.full(shape, float("nan"), dtype=torch.float32, device=dev)
            _lib.check(_call(L.ipb_match_template_device_noalloc, di, dt, dm, method, precision,
                             got, stream))
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))


def test_noalloc_rejects_problems_above_its_fixed_scratch():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    image = torch.zeros((3000, 3000), dtype=torch.uint8, device=dev)  # 72 MB integral image
    template = torch.zeros((16, 16), dtype=torch.uint8, device=dev)
    out = torch.empty((2985, 2985), dtype=torch.float32, device=dev)
    st = _call(L.ipb_match_template_device_noalloc, image, template, None, 0, EXACT_FP64, out, None)
    assert st == _lib.ERR_INVALID_ARGUMENT
    msg = L.ipb_last_error_message().decode()
    assert "fixed maximum" in msg and "bytes" in msg
