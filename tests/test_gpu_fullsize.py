"""Full-size parity of the two batched workloads the benchmark times.

* Uneven pairs: the exact 256-pair draw the benchmark runs
  (synthetic.uneven_pairs(seed=3): image sides log-uniform 256..4096, template
  sides 8..128, methods 0..3), as one batch plan with find_extremes fused.
  Every pair's fused extremes must equal the oracle's find_extremes of the
  oracle's map (src/template_matching.rs:479-511, first occurrence), and the
  full maps of at least 16 pairs (the largest image, the largest template,
  every method, the narrowest templates, seeded picks) must equal the oracle's
  bit for bit (match_template, :78-92).
* Many templates: the 4096 x 4096 value-noise scene with its 512 templates of
  32 x 32 (synthetic.value_noise_scene(), the benchmark's draw),
  CrossCorrelationNormalized (:271-293) in one launch with find_extremes
  fused: every template's map on two seeded 64-row bands and eight
  templates' full maps bit for bit, and all 512 fused extremes against the
  oracle's.

The oracle is the fast exact form (oracle/tm_oracle.c tmo_many_exact_fast),
which tests/test_oracle_fast.py pins to the plain restatement.
"""

import numpy as np
import pytest

from imageproc_b200 import synthetic
from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _ext_tuple(e):
    return (np.float32(e.max_value), np.float32(e.min_value), tuple(e.max_value_location),
            tuple(e.min_value_location))


def _same_extremes(got, exp):
    gmx, gmn, gmxl, gmnl = got
    emx, emn, emxl, emnl = exp
    return (bits(np.float32(gmx)) == bits(np.float32(emx)) and bits(np.float32(gmn)) == bits(np.float32(emn))
            and gmxl == emxl and gmnl == emnl)


def _full_map_picks(pairs, n_picks=16, seed=17):
    """Indices of the pairs whose whole maps are compared."""
    area = [i.size for i, _, _ in pairs]
    tarea = [t.size for _, t, _ in pairs]
    picks = {int(np.argmax(area)), int(np.argmax(tarea))}
    for m in range(4):  # every method
        picks.add(next(k for k, p in enumerate(pairs) if p[2] == m))
    # the narrowest templates (8..15 columns: half of the first 32-byte K step
    # of the tensor-core kernel) and a wide one
    picks.add(next(k for k, (_, t, _) in enumerate(pairs) if t.shape[1] < 16))
    picks.add(next(k for k, (_, t, _) in enumerate(pairs) if t.shape[1] >= 64))
    g = np.random.default_rng(seed)
    for k in g.permutation(len(pairs)):
        if len(picks) >= n_picks:
            break
        picks.add(int(k))
    return sorted(picks)


def test_uneven_pairs_full_draw():
    import torch

    from imageproc_b200 import device

    pairs = synthetic.uneven_pairs(seed=3)
    assert len(pairs) == 256
    items = [(torch.from_numpy(i).cuda(), torch.from_numpy(t).cuda(), m) for i, t, m in pairs]
    batch = device.Batch(items, extremes=True)
    plan = device.BatchPlan(batch, tm.Precision.ExactFp64)
    info = plan.info()
    assert info["tensor_pairs"] > 0
    plan.launch()
    torch.cuda.synchronize()
    got_ext = [_ext_tuple(e) for e in batch.extremes_host()]
    picks = set(_full_map_picks(pairs))
    assert len(picks) >= 16
    bad_ext, bad_maps = [], []
    for k, (image, template, method) in enumerate(pairs):
        want_map = k in picks
        exp_map, exp_ext = O.match_exact_fast(image, template, method, precision=0,
                                              want_map=want_map)
        if not _same_extremes(got_ext[k], exp_ext):
            bad_ext.append((k, got_ext[k], exp_ext))
        if want_map:
            got = batch.outs[k].cpu().numpy()
            if not np.array_equal(bits(got), bits(exp_map)):
                bad_maps.append((k, int((bits(got) != bits(exp_map)).sum())))
    plan.close()
    assert not bad_ext, f"{len(bad_ext)} extremes differ, first: {bad_ext[:3]}"
    assert not bad_maps, f"maps differ (pair, differing scores): {bad_maps}"


def test_many_templates_full_scene():
    import torch

    from imageproc_b200 import device

    image, templates, locs = synthetic.value_noise_scene()
    n, h, w = templates.shape
    assert (image.shape, n, h, w) == ((4096, 4096), 512, 32, 32)
    Ho, Wo = image.shape[0] - h + 1, image.shape[1] - w + 1
    method = tm.MatchTemplateMethod.CrossCorrelationNormalized
    di = torch.from_numpy(image).cuda()
    dt = torch.from_numpy(templates).cuda()
    out, ext = device.match_templates_device(di, dt, method, extremes=True)
    torch.cuda.synchronize()
    assert out.shape == (Ho, Wo, n)

    # every template's map on two seeded 64-row bands
    g = np.random.default_rng(2024)
    for y0 in sorted(int(v) for v in g.choice(Ho - 64, size=2, replace=False)):
        exp, _ = O.many_exact_fast(image, templates, int(method), rows=(y0, y0 + 64),
                                   want_maps=True)
        got = out[y0:y0 + 64].permute(2, 0, 1).contiguous().cpu().numpy()
        diff = bits(got) != bits(exp)
        assert not diff.any(), f"band y0={y0}: {int(diff.sum())} scores differ"

    # eight templates' full maps (the first, the last, six seeded)
    for t in sorted({0, n - 1, *(int(v) for v in g.choice(n, size=6, replace=False))}):
        exp, _ = O.match_exact_fast(image, templates[t], int(method), precision=0)
        got = out[:, :, t].contiguous().cpu().numpy()
        diff = bits(got) != bits(exp)
        assert not diff.any(), f"template {t}: {int(diff.sum())} scores differ"
    del out
    torch.cuda.empty_cache()

    # all 512 fused extremes against the oracle's find_extremes of every map
    _, exp_ext = O.many_exact_fast(image, templates, int(method), want_maps=False)
    bad = [(t, _ext_tuple(ext[t]), exp_ext[t]) for t in range(n)
           if not _same_extremes(_ext_tuple(ext[t]), exp_ext[t])]
    assert not bad, f"{len(bad)} of {n} extremes differ, first: {bad[:3]}"
    # and the scene is what the benchmark reports on: the best match of most
    # templates is their own crop
    hits = sum(1 for t in range(n) if tuple(ext[t].max_value_location) == tuple(locs[t]))
    assert hits >= n * 0.9
