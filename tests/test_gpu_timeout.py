"""Failure detection on the GPU without a fault: the tensor-core kernels'
bounded waits are made to run out, and the call must report IPB_ERR_TIMEOUT
while the context stays usable.

Two test hooks do it: ipb_debug_stall_pipelines makes the MMA-issuing warp of
each tensor-core kernel first wait on an mbarrier that nothing arrives at (a
flag that nothing sets), and ipb_debug_set_pipeline_wait_ns shortens the
per-tile budget of every bounded wait to 100 us so the test stays short. The
kernel then records its launch tag in the error word, stops its pipeline,
waits (with the full 2 s budget) for the tensor-core work it issued, frees its
tensor memory and exits; nothing faults, traps or spins without a limit. The
next call, with the hooks off, must run on the same context and be exact.
"""

import numpy as np
import pytest

from imageproc_b200 import _lib, synthetic
from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


BUDGET_NS = 100_000


def _stall(L, on):
    L.ipb_debug_set_pipeline_wait_ns(BUDGET_NS if on else 0)
    L.ipb_debug_stall_pipelines(1 if on else 0)


@pytest.fixture
def tiny_budget():
    L = _lib.lib()
    yield L
    _stall(L, False)  # default budget and no stall again, whatever happened


def test_single_template_wait_runs_out_then_context_recovers(tiny_budget):
    L = tiny_budget
    image, template, mask, _ = synthetic.blob_scene(W=700, H=400, tw=64, th=48, seed=77)
    tm.set_precision(tm.Precision.ExactFp64)
    tm.set_path(tm.Path.Auto)
    for masked in (False, True):
        _stall(L, True)
        with pytest.raises(_lib.DeviceError, match=r"status 9\].*timed out"):
            if masked:
                tm.match_template_with_mask(image, template, 3, mask)
            else:
                tm.match_template(image, template, 0)
        _stall(L, False)
        # tensor memory was freed and the context is usable: two exact calls
        for _ in range(2):
            if masked:
                got = tm.match_template_with_mask(image, template, 3, mask)
                exp = O.match_exact(image, template, 3, mask, precision=0)
            else:
                got = tm.match_template(image, template, 0)
                exp = O.match_exact(image, template, 0, None, precision=0)
            assert np.array_equal(bits(got), bits(exp))


def test_many_templates_wait_runs_out_then_context_recovers(tiny_budget):
    import torch

    from imageproc_b200 import device
    L = tiny_budget
    image, templates, _ = synthetic.value_noise_scene(W=512, H=384, n_templates=130, t=32, seed=9)
    di = torch.from_numpy(image).cuda()
    dt = torch.from_numpy(templates).cuda()
    _stall(L, True)
    device.match_templates_device(di, dt, 3, extremes=False)  # enqueues; the failure shows at the next sync
    torch.cuda.synchronize()
    _stall(L, False)
    # the next synchronous call of this thread's context reports the earlier launch's timeout ...
    small, tpl = image[:100, :200].copy(), templates[0]
    with pytest.raises(_lib.DeviceError, match=r"status 9\]"):
        tm.match_template(small, tpl, 2)
    # ... once, and then every call is exact again
    got = tm.match_template(small, tpl, 2)
    assert np.array_equal(bits(got), bits(O.match_exact(small, tpl, 2, None, precision=0)))
    out, _ = device.match_templates_device(di, dt, 3, extremes=False)
    torch.cuda.synchronize()
    k = 77
    exp = O.match_exact(image, templates[k], 3, None, precision=0)
    assert np.array_equal(bits(out[:, :, k].cpu().numpy()), bits(exp))
