"""Page-locked host buffers (ipb_host_alloc / ipb_host_free) and the host API's
score maps, which are allocated from them."""

import gc

import numpy as np
import pytest

from imageproc_b200 import _lib
from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_host_alloc_reuses_freed_blocks():
    L = _lib.lib()
    p = L.ipb_host_alloc(3 << 20)
    assert p
    L.ipb_host_free(p)
    q = L.ipb_host_alloc(3 << 20)
    assert q == p  # the cached block comes back
    L.ipb_host_free(q)
    L.ipb_host_free(None)  # no-op
    L.ipb_host_cache_release()  # the cached block goes back to the driver
    r = L.ipb_host_alloc(3 << 20)
    assert r
    L.ipb_host_free(r)


def test_host_api_scores_come_from_the_cache_and_are_correct():
    # start from an empty cache: blocks that earlier calls left in it would
    # otherwise be handed out first
    _lib.lib().ipb_host_cache_release()
    g = np.random.default_rng(3)
    image = g.integers(0, 256, (300, 400), dtype=np.uint8)
    template = g.integers(0, 256, (24, 20), dtype=np.uint8)
    addrs = set()
    for method in tm.MatchTemplateMethod:
        out = tm.match_template(image, template, method)
        addrs.add(out.ctypes.data)
        exp = O.match_exact(image, template, method, None, precision=0)
        assert np.array_equal(out.view(np.uint32), exp.view(np.uint32))
    # a view keeps the block alive
    view = out[5:10].copy()
    part = out[5:10]
    del out
    gc.collect()
    assert np.array_equal(part, view)
    # once the last views are gone the blocks return to the cache: the next
    # allocation of that size gets one of the score maps' page-locked blocks
    del part
    gc.collect()
    L = _lib.lib()
    p = L.ipb_host_alloc(277 * 381 * 4)
    assert p in addrs
    L.ipb_host_free(p)
