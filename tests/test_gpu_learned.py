"""The proposal network on the GPU: its gradients against the FP64 oracle,
training, and the propose-verify-certify pipeline against the exhaustive
answers (the oracle's SumOfSquaredErrors minimum, src/template_matching.rs:
214-228 with find_extremes :479-511).

Tolerances: the GPU accumulates in fp32 and keeps the backward pass's
activation gradients in bf16; the oracle computes the same network (the same
bf16 roundings in the forward pass) in FP64. Loss: 2e-3 relative. Gradients:
relative L2 error <= 0.1 and cosine >= 0.995 per layer (every backward
convolution rounds its output to bf16). Answers: exact.
"""

import numpy as np
import pytest

from imageproc_b200 import learned, synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _params(seed):
    # He-normal weights scaled by 0.7 per layer, small biases: logits of a few
    # units, so the softmax is neither flat nor saturated
    p = learned.init_params(seed)
    g = np.random.default_rng(50 + seed)
    off = 0
    for cin in (1, 32, 32, 32, 32):
        p[off:off + 32 * cin * 9] *= 0.7
        off += 32 * cin * 9
        p[off:off + 32] = g.normal(0, 0.05, 32).astype(np.float32)
        off += 32
    return p


def _layer_slices():
    out, off = [], 0
    for cin in (1, 32, 32, 32, 32):
        n = 32 * cin * 9
        out.append((f"W{len(out) // 2 + 1}", slice(off, off + n)))
        out.append((f"b{len(out) // 2 + 1}", slice(off + n, off + n + 32)))
        off += n + 32
    return out


@pytest.mark.parametrize("seed,n,side,t", [(0, 4, 32, 4), (1, 3, 64, 5)])
def test_gradients_match_oracle(seed, n, side, t):
    import torch
    g = np.random.default_rng(seed)
    scene = synthetic.rect_scene(W=512, H=512, n_rects=20, n_templates=0, seed=300 + seed)[0]
    ys = g.integers(0, (512 - side) // 4, n) * 4
    xs = g.integers(0, (512 - side) // 4, n) * 4
    scenes = np.stack([scene[y:y + side, x:x + side] for y, x in zip(ys, xs)])
    templates = np.stack([scene[y:y + 48, x:x + 48] for y, x in
                          zip(g.integers(0, 464, t), g.integers(0, 464, t))])
    P = n * (side // 4) ** 2
    pos = g.integers(0, P, t).astype(np.int64)
    params = _params(seed)
    net = learned.ProposalNet(params)
    loss, grads = net.gradients(torch.from_numpy(scenes).cuda(), torch.from_numpy(templates).cuda(),
                                torch.from_numpy(pos).cuda())
    ref_loss, ref = O.learned_loss_grad(params, scenes, templates, pos, bf16=True)
    assert abs(loss - ref_loss) <= 2e-3 * abs(ref_loss), (loss, ref_loss)
    for name, sl in _layer_slices():
        a, b = grads[sl].astype(np.float64), ref[sl]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        cos = float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))
        # each data-gradient convolution rounds its output to bf16
        assert rel <= 0.1 and cos >= 0.995, (name, rel, cos)


@pytest.mark.parametrize("H,W", [(64, 96), (200, 540), (12 * 4, 12 * 4)])
def test_features_tensor_cores_match_oracle(H, W):
    # the 32-channel layers on tcgen05 (query path) and on mma.sync (training
    # path) against the FP64 oracle of the same network: the activations are
    # bf16, so a value differs where an fp32 sum straddles a rounding boundary
    # and the difference propagates through the later layers; tolerance: max
    # error 3e-2 and mean error 1e-3 of the largest feature
    import torch
    params = _params(2)
    net = learned.ProposalNet(params)
    g = np.random.default_rng(H + W)
    image = g.integers(0, 256, (H, W), dtype=np.uint8)
    di = torch.from_numpy(image).cuda()
    tc = net.features(di, kernel=0).cpu().numpy().astype(np.float64)
    mma = net.features(di, kernel=1).cpu().numpy().astype(np.float64)
    ref = O.learned_features(params, image[None])[0]
    scale = np.abs(ref).max()
    for got in (tc, mma):
        err = np.abs(got - ref)
        assert err.max() <= 3e-2 * scale, err.max() / scale
        assert err.mean() <= 1e-3 * scale, err.mean() / scale
    assert np.abs(tc - mma).mean() <= 1e-3 * scale


def test_training_reduces_the_loss():
    import torch
    scene = synthetic.rect_scene(W=2048, H=2048, n_rects=60, n_templates=0, seed=1500)[0]
    scenes = torch.from_numpy(scene[None]).cuda()
    net = learned.ProposalNet(seed=3)
    losses = learned.train(net, scenes, pairs=64 * 120, batch=64, lr=2e-3, seed=4, log=None)
    first, last = np.mean(losses[:10]), np.mean(losses[-10:])
    assert np.isfinite(losses).all()
    assert last < 0.7 * first, (first, last)


def _exact_answers(image, templates):
    _, ext = O.many_exact_fast(image, templates, 0, want_maps=False)
    return [(e[1], e[3]) for e in ext]  # (min value, (x, y))


def _check_exact(answers, exact):
    bad = []
    for k, (a, (v, loc)) in enumerate(zip(answers, exact)):
        if not (np.float32(a.value).view(np.uint32) == np.float32(v).view(np.uint32) and a.location == tuple(loc)):
            bad.append((k, a, v, loc))
    return bad


@pytest.mark.parametrize("trained", [False, True])
def test_propose_and_match_equals_exhaustive(trained):
    import torch
    image, templates, _ = synthetic.rect_scene(W=2048, H=2048, n_rects=60, n_templates=64, seed=77)
    net = learned.ProposalNet.trained() if trained else learned.ProposalNet(seed=11)
    di, dt = torch.from_numpy(image).cuda(), torch.from_numpy(templates).cuda()
    answers = net.propose_and_match(di, dt)
    exact = _exact_answers(image, templates)
    bad = _check_exact(answers, exact)
    assert not bad, bad[:4]
    # every path gives the exact answer; a template answered without the
    # exhaustive kernel had a certificate
    paths = np.bincount([a.path for a in answers], minlength=3)
    assert paths.sum() == 64


def test_trained_network_gains_over_untrained():
    import torch
    image, templates, _ = synthetic.rect_scene(W=2048, H=2048, n_rects=60, n_templates=64, seed=78)
    di, dt = torch.from_numpy(image).cuda(), torch.from_numpy(templates).cuda()
    trained = learned.ProposalNet.trained().propose_and_match(di, dt)
    untrained = learned.ProposalNet(seed=12).propose_and_match(di, dt)
    ok_t = sum(a.path == 0 for a in trained) / 64
    ok_u = sum(a.path == 0 for a in untrained) / 64
    assert ok_t >= 0.8 and ok_t >= ok_u + 0.3, (ok_t, ok_u)


def test_ablation_network_and_pyramid_proposals():
    # the same verification, certification and fallback fed by the trained
    # network (with the 0.1 margin gate, and with the certificate alone) or by
    # coarse-pyramid proposals: every answer exact; dropping the margin gate
    # only moves templates from the fallback to the certificate; the rates
    # themselves are reported by bench.py (learned.ablation_pyramid)
    import torch
    image, templates, _ = synthetic.rect_scene(W=2048, H=2048, n_rects=60, n_templates=64, seed=79)
    di, dt = torch.from_numpy(image).cuda(), torch.from_numpy(templates).cuda()
    exact = _exact_answers(image, templates)
    trained = learned.ProposalNet.trained()
    net = trained.propose_and_match(di, dt)
    net0 = trained.propose_and_match(di, dt, min_margin=0.0)
    pyr = learned.match_proposals(di, dt, learned.pyramid_origins(di, dt))
    for answers in (net, net0, pyr):
        assert not _check_exact(answers, exact)
    ok = [sum(a.path == 0 for a in answers) / 64 for answers in (net, net0, pyr)]
    assert ok[1] >= ok[0] and min(ok) >= 0.8, ok
    assert all(a.path in (0, 2) for a in net0 + pyr)  # no margin gate on these


def test_rejects_unsupported_queries():
    import torch
    net = learned.ProposalNet(seed=1)
    image = torch.zeros((256, 256), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError, match="48 x 48"):
        net.propose_and_match(image, torch.zeros((2, 32, 32), dtype=torch.uint8, device="cuda"))
    with pytest.raises(ValueError, match="multiples of 32"):
        net.propose_and_match(torch.zeros((250, 256), dtype=torch.uint8, device="cuda"),
                              torch.zeros((2, 48, 48), dtype=torch.uint8, device="cuda"))
    shifted = torch.zeros(256 * 256 + 16, dtype=torch.uint8, device="cuda")[1:1 + 256 * 256].view(256, 256)
    with pytest.raises(ValueError, match="16-byte aligned"):
        net.propose_and_match(shifted, torch.zeros((2, 48, 48), dtype=torch.uint8, device="cuda"))
