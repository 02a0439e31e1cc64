"""Batched matching (one persistent launch per tensor-core group, CUDA graphs)
against the oracle, including the fused find_extremes.

Bar: every score map bit-exact against the oracle's exact-sum epilogue, every
extremes record equal to the oracle's find_extremes of that map (first
occurrence on ties, src/template_matching.rs:494-503).
"""

import numpy as np
import pytest

from imageproc_b200 import _lib, synthetic
from imageproc_b200 import template_matching as tm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _mixed_items(seed, n):
    """Uneven pairs: tensor-core shapes of every row width, CUDA-core shapes
    (templates narrower than 8 or general masks), binary masks, all methods."""
    g = np.random.default_rng(seed)
    items = []
    for k in range(n):
        H, W = int(g.integers(40, 400)), int(g.integers(40, 700))
        h = int(g.integers(1, min(H, 120) + 1))
        w = int(g.integers(4, min(W, 200) + 1))
        image = g.integers(0, 256, (H, W), dtype=np.uint8)
        if k % 7 == 3:
            image[:] = 200  # flat: every score ties, extremes at the first pixel
        template = g.integers(0, 256, (h, w), dtype=np.uint8)
        method = int(g.integers(0, 4))
        kind = k % 3
        mask = None
        if kind == 1:
            mask = (g.random((h, w)) < 0.8).astype(np.uint8)
        items.append((image, template, method, mask))
    return items


def _to_device(items):
    import torch
    dev = []
    for image, template, method, mask in items:
        t = (torch.from_numpy(image).cuda(), torch.from_numpy(template).cuda(), method)
        if mask is not None:
            t = t + (torch.from_numpy(mask).cuda(),)
        dev.append(t)
    return dev


def _check(items, outs, extremes):
    for k, ((image, template, method, mask), out, ex) in enumerate(zip(items, outs, extremes)):
        got = out.cpu().numpy()
        exp = O.match_exact(image, template, method, mask, precision=0)
        bad = np.argwhere(bits(got) != bits(exp))
        assert bad.size == 0, (k, image.shape, template.shape, method, mask is not None, bad[:3])
        mx, mn, mxl, mnl = O.find_extremes(exp)
        assert (ex.max_value, ex.min_value, ex.max_value_location, ex.min_value_location) == \
            (float(mx), float(mn), mxl, mnl), k


@pytest.mark.parametrize("seed", [1, 2])
def test_batch_mixed_pairs_bit_exact_with_fused_extremes(seed):
    from imageproc_b200 import device
    items = _mixed_items(seed, 20)
    batch = device.Batch(_to_device(items))
    batch.run()
    _check(items, batch.outs, batch.extremes_host())


def test_batch_plan_graph_replay():
    import torch

    from imageproc_b200 import device
    items = _mixed_items(7, 12)
    batch = device.Batch(_to_device(items))
    plan = device.BatchPlan(batch)
    info = plan.info()
    assert info["tensor_pairs"] >= 1 and info["kernels"] >= 1
    n0 = _lib.launch_count()
    for _ in range(2):
        for o in batch.outs:
            o.fill_(float("nan"))
        batch.extremes.zero_()
        plan.launch()
        torch.cuda.synchronize()
        _check(items, batch.outs, batch.extremes_host())
    assert _lib.launch_count() - n0 == 2 * info["kernels"]
    plan.close()


def test_batch_groups_side_by_side_claim_every_tile_once():
    # an unmasked and a binary-mask group, each with more tiles than SMs, so
    # CTAs claim tiles from the launch's counter while the two launches run on
    # two streams; run four times (a one-off plan, the plan's graph, the plan
    # enqueued directly with its kernels timed, the graph again) over NaN-filled
    # outputs, so a tile skipped or a counter left armed shows as a mismatch
    import torch

    from imageproc_b200 import device
    g = np.random.default_rng(11)
    image = g.integers(0, 256, (640, 1024), dtype=np.uint8)
    template = g.integers(0, 256, (40, 48), dtype=np.uint8)
    mask = (g.random((40, 48)) < 0.8).astype(np.uint8)
    items = [(image, template, m, None) for m in range(4)] + [(image, template, m, mask) for m in range(4)]
    batch = device.Batch(_to_device(items))
    plan = device.BatchPlan(batch)
    assert plan.info()["tensor_pairs"] == 8
    expected = [O.match_exact(image, template, m, mk, precision=0) for image, template, m, mk in items]
    _lib.profile_collect()  # drop stats left by earlier calls
    for launch, timed in ((batch.run, False), (plan.launch, False), (plan.launch, True), (plan.launch, False)):
        for o in batch.outs:
            o.fill_(float("nan"))
        batch.extremes.zero_()
        _lib.profile_enable(timed)  # timed: the plan's launches enqueued directly, not as its graph
        try:
            launch()
            torch.cuda.synchronize()
        finally:
            _lib.profile_enable(False)
        for k, (out, exp) in enumerate(zip(batch.outs, expected)):
            bad = np.argwhere(bits(out.cpu().numpy()) != bits(exp))
            assert bad.size == 0, (k, timed, bad[:3])
    assert _lib.profile_collect()["umma_i8"]["launches"] == 2  # the two side-by-side launches, timed as one span
    plan.close()


def test_batch_of_more_problems_than_fit_in_kernel_parameters():
    # > 8 tensor pairs of one group: problem descriptors come from device memory
    from imageproc_b200 import device
    g = np.random.default_rng(3)
    items = []
    for k in range(13):
        H, W = int(g.integers(64, 300)), int(g.integers(64, 500))
        image = g.integers(0, 256, (H, W), dtype=np.uint8)
        template = g.integers(0, 256, (int(g.integers(8, 60)), int(g.integers(33, 64))), dtype=np.uint8)
        items.append((image, template, k % 4, None))
    batch = device.Batch(_to_device(items))
    plan = device.BatchPlan(batch)
    assert plan.info()["tensor_pairs"] == 13
    plan.launch()
    import torch
    torch.cuda.synchronize()
    _check(items, batch.outs, batch.extremes_host())
    plan.close()


def test_uneven_pairs_workload_reduced():
    # the batched workload's generator at reduced image sides, all pairs checked
    from imageproc_b200 import device
    pairs = synthetic.uneven_pairs(n=24, seed=3, lo=128, hi=768)
    items = [(im, tp, m, None) for im, tp, m in pairs]
    batch = device.Batch(_to_device(items))
    batch.run()
    _check(items, batch.outs, batch.extremes_host())


def test_batch_rejects_invalid_pair_before_any_work():
    import torch

    from imageproc_b200 import device
    img = torch.zeros((10, 10), dtype=torch.uint8, device="cuda")
    ok_t = torch.zeros((3, 3), dtype=torch.uint8, device="cuda")
    bad_t = torch.zeros((3, 12), dtype=torch.uint8, device="cuda")
    batch = device.Batch([(img, ok_t, 0), (img, bad_t, 0)])
    batch.outs[0].fill_(-1.0)
    with pytest.raises(tm.Panic, match="^pair 1: image width must be greater than or equal to template width$"):
        batch.run()
    torch.cuda.synchronize()
    assert (batch.outs[0] == -1.0).all()


def test_batch_tuner_persists_choices_and_replays_rearm_extremes(tmp_path, monkeypatch):
    # the default group tuner times each natural group's row width and tile
    # height, persists the choice, and a later plan reads it back; results
    # stay bit-exact whatever the choice, and each replay re-arms the fused
    # extremes (the second launch sees new image content)
    import torch

    from imageproc_b200 import device
    L = _lib.lib()
    L.ipb_batch_tuning_reset.argtypes = []
    L.ipb_batch_tuning_reset.restype = None
    f = tmp_path / "tuning.txt"
    monkeypatch.setenv("IPB_TUNING_FILE", str(f))
    monkeypatch.delenv("IPB_AUTOTUNE", raising=False)
    L.ipb_batch_tuning_reset()
    pairs = synthetic.uneven_pairs(n=24, seed=7, lo=128, hi=768)
    items = [(im, tp, m, None) for im, tp, m in pairs]
    dev_items = _to_device(items)
    batch = device.Batch(dev_items)
    plan = device.BatchPlan(batch)
    info = plan.info()
    assert info["kernels"] == len(info["launches"]) + 1  # tensor launches + the extremes finish
    assert info["tensor_pairs"] == len(items)
    # "group2 ks0 masked h8 wlog mlog set ks nt n": the group key (natural row
    # width, mask kind, template height, sizes, largest set the pairs form)
    # and the choice (row width, tile height, problems per set)
    groups = [ln.split() for ln in f.read_text().splitlines() if ln.startswith("group2 ")]
    assert groups, "group decisions persisted"
    plan.launch()
    torch.cuda.synchronize()
    _check(items, batch.outs, batch.extremes_host())
    # new content in every image, same plan: extremes from this launch only
    g = np.random.default_rng(11)
    new_items = []
    for (image, template, method, mask), d in zip(items, dev_items):
        fresh = g.integers(0, 256, image.shape, dtype=np.uint8)
        d[0].copy_(torch.from_numpy(fresh))
        new_items.append((fresh, template, method, mask))
    plan.launch()
    torch.cuda.synchronize()
    _check(new_items, batch.outs, batch.extremes_host())
    plan.close()
    # a persisted choice is read back: force 64-row tiles at the natural width
    f.write_text("".join(f"group2 {k[1]} {k[2]} {k[3]} {k[4]} {k[5]} {k[6]} {k[1]} 64 1\n" for k in groups))
    L.ipb_batch_tuning_reset()
    plan2 = device.BatchPlan(batch)
    info2 = plan2.info()
    assert {g2["tile_rows"] for g2 in info2["launches"]} == {64}
    plan2.launch()
    torch.cuda.synchronize()
    _check(new_items, batch.outs, batch.extremes_host())
    plan2.close()
    L.ipb_batch_tuning_reset()


def _shared_image_items(seed):
    """Pairs that share images: per image, classes of 1..8 pairs with one
    template size (own template content, methods, binary masks or none), a
    class that repeats one template over all four methods, a second template
    size on the same image, and binary-mask classes that share one mask
    buffer. Odd image sizes, so that tiles are ragged at both edges."""
    g = np.random.default_rng(seed)
    items = []
    for H, W, sizes in [(301, 517, [(64, 64, 8), (20, 33, 3)]), (143, 260, [(48, 48, 5)]),
                        (90, 1100, [(17, 130, 2), (9, 8, 4)]), (260, 260, [(64, 64, 1)])]:
        image = g.integers(0, 256, (H, W), dtype=np.uint8)
        for h, w, count in sizes:
            for masked in (False, True):
                if masked and w > 128:
                    continue
                for _ in range(count):
                    template = g.integers(0, 256, (h, w), dtype=np.uint8)
                    mask = (g.random((h, w)) < 0.8).astype(np.uint8) if masked else None
                    items.append((image, template, int(g.integers(0, 4)), mask))
        template = g.integers(0, 256, (32, 40), dtype=np.uint8)
        for method in range(4):  # one template, every method
            items.append((image, template, method, None))
        # binary-mask pairs sharing one mask buffer (their sets compute the
        # common Y = sum I^2 m once): mixed methods, then CrossCorrelation
        # alone (no Y at all)
        for count, methods in ((6, None), (3, 2)):
            mask = (g.random((24, 36)) < 0.7).astype(np.uint8)
            for _ in range(count):
                template = g.integers(0, 256, (24, 36), dtype=np.uint8)
                method = int(g.integers(0, 4)) if methods is None else methods
                items.append((image, template, method, mask))
        template = g.integers(0, 256, (24, 36), dtype=np.uint8)
        for method in range(4):  # one template and one mask, every method
            items.append((image, template, method, mask))
    return items


def _to_device_shared(items):
    """Device tensors with one copy per distinct host array (pairs that share
    an image share its device buffer, so the planner can form sets)."""
    import torch
    cache = {}

    def dev(a):
        if id(a) not in cache:
            cache[id(a)] = torch.from_numpy(a).cuda()
        return cache[id(a)]
    out = []
    for image, template, method, mask in items:
        t = (dev(image), dev(template), method)
        if mask is not None:
            t = t + (dev(mask),)
        out.append(t)
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_pairs_sharing_images_form_sets_bit_exact(precision):
    """Pairs on one image with one template size are computed together
    (sets of up to four share the image's A rows; each keeps its own
    template side, accumulators and epilogue): every map and extremes record
    must equal the oracle's, for both exact precisions, and a replayed plan
    must give the same again."""
    import torch

    from imageproc_b200 import device
    items = _shared_image_items(11 + precision)
    batch = device.Batch(_to_device_shared(items))
    plan = device.BatchPlan(batch, precision)
    for _ in range(2):
        for out in batch.outs:
            out.fill_(-1.0)
        plan.launch()
        torch.cuda.synchronize()
        ex = batch.extremes_host()
        for k, ((image, template, method, mask), out, e) in enumerate(zip(items, batch.outs, ex)):
            got = out.cpu().numpy()
            exp = O.match_exact(image, template, method, mask, precision=precision)
            bad = np.argwhere(bits(got) != bits(exp))
            assert bad.size == 0, (k, image.shape, template.shape, method, mask is not None, bad[:3])
            mx, mn, mxl, mnl = O.find_extremes(exp)
            assert (e.max_value, e.min_value, e.max_value_location, e.min_value_location) == \
                (float(mx), float(mn), mxl, mnl), k
