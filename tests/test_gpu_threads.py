"""The host entry points from several threads at once, as the reference's
functions allow (they are Sync, src/template_matching.rs:165-168): each
calling thread gets its own context and stream, so concurrent calls of
different shapes and methods must each return their own exact result."""

import threading

import numpy as np
import pytest

from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu
M = tm.MatchTemplateMethod


@pytest.fixture
def exact_fp64():
    old = tm.get_precision()
    tm.set_precision(tm.Precision.ExactFp64)
    yield
    tm.set_precision(old)


def test_concurrent_calls_from_threads(exact_fp64):
    g = np.random.default_rng(17)
    jobs = []
    for k in range(12):
        H, W = int(g.integers(60, 300)), int(g.integers(60, 300))
        h, w = int(g.integers(8, 40)), int(g.integers(16, 48))
        image = g.integers(0, 256, (H, W), dtype=np.uint8)
        template = g.integers(0, 256, (h, w), dtype=np.uint8)
        mask = (g.random((h, w)) < 0.7).astype(np.uint8) if k % 3 == 0 else None
        jobs.append((image, template, M(k % 4), mask))
    expected = [O.match_exact(i, t, m, mk, precision=0) for i, t, m, mk in jobs]
    results = [None] * len(jobs)
    errors = []

    def run(slot):
        try:
            for _ in range(5):  # repeat so calls interleave
                for j in range(slot, len(jobs), 4):
                    i, t, m, mk = jobs[j]
                    out = tm.match_template(i, t, m) if mk is None else tm.match_template_with_mask(i, t, m, mk)
                    if results[j] is None:
                        results[j] = out.copy()
                    elif not np.array_equal(results[j].view(np.uint32), out.view(np.uint32)):
                        errors.append(("nondeterministic", j))
        except Exception as e:  # surfaced below
            errors.append(repr(e))

    threads = [threading.Thread(target=run, args=(s,)) for s in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for j, (got, exp) in enumerate(zip(results, expected)):
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), j
