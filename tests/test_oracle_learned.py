"""The proposal network's FP64 CPU oracle (oracle/learned_oracle.c), pinned
by central finite differences of its own loss (pure FP64, bf16 roundings off):
its analytic gradients are what the GPU training kernels are checked against.
"""

import numpy as np
import pytest

from imageproc_b200 import learned
from oracle import oracle as O


def _batch(seed, n=2, side=16, t=2):
    g = np.random.default_rng(seed)
    scenes = g.integers(0, 256, (n, side, side), dtype=np.uint8)
    templates = g.integers(0, 256, (t, 48, 48), dtype=np.uint8)
    P = n * (side // 4) ** 2
    pos = g.integers(0, P, t).astype(np.int64)
    return scenes, templates, pos


def test_parameter_layout_matches_the_library():
    assert learned.N_PARAMS == 32 * 9 + 32 + 4 * (32 * 32 * 9 + 32)
    p = learned.init_params(3)
    assert p.shape == (learned.N_PARAMS,) and p.dtype == np.float32
    Ws, bs = O._lo_split(p)
    assert [w.shape for w in Ws] == [(32, 1, 3, 3)] + [(32, 32, 3, 3)] * 4
    assert all(np.all(b == 0) for b in bs)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_gradients_match_finite_differences(seed):
    scenes, templates, pos = _batch(seed)
    params = learned.init_params(seed).astype(np.float64)
    # small non-zero biases so every bias gradient is exercised
    g = np.random.default_rng(100 + seed)
    Ws, bs = O._lo_split(params)
    off = 0
    for w in Ws:
        off += w.size
        params[off:off + 32] = g.normal(0, 0.05, 32)
        off += 32
    loss, grads = O.learned_loss_grad(params, scenes, templates, pos, bf16=False)
    assert np.isfinite(loss) and loss > 0
    # coordinates: a few weights and biases of every layer
    idx = []
    off = 0
    for w in Ws:
        idx += list(off + g.choice(w.size, 4, replace=False))
        off += w.size
        idx += list(off + g.choice(32, 2, replace=False))
        off += 32
    eps = 1e-5
    bad = []
    for i in idx:
        p1 = params.copy()
        p1[i] += eps
        p2 = params.copy()
        p2[i] -= eps
        fd = (O.learned_loss_grad(p1, scenes, templates, pos, bf16=False)[0] -
              O.learned_loss_grad(p2, scenes, templates, pos, bf16=False)[0]) / (2 * eps)
        if abs(fd - grads[i]) > 1e-5 + 1e-4 * abs(fd):
            bad.append((int(i), fd, grads[i]))
    assert not bad, bad


def test_oracle_loss_at_zero_weights():
    # all logits 0: each template's loss is log(P) - log(|N_t|), N_t the 3 x 3
    # neighbourhood of its positive clipped to the crop
    scenes, templates, pos = _batch(5, n=3, side=24, t=3)
    pos[0] = 0  # a corner: a neighbourhood of 4
    params = np.zeros(learned.N_PARAMS)
    loss, grads, z = O.learned_loss_grad(params, scenes, templates, pos, bf16=True, want_logits=True)
    assert np.allclose(z, 0.0)
    hs = ws = 24 // 4
    sizes = []
    for p in pos:
        y, x = (p % (hs * ws)) // ws, p % ws
        sizes.append((min(y + 1, hs - 1) - max(y - 1, 0) + 1) * (min(x + 1, ws - 1) - max(x - 1, 0) + 1))
    assert sizes[0] == 4
    exp = np.mean([np.log(z.shape[1]) - np.log(k) for k in sizes])
    assert abs(loss - exp) < 1e-12
