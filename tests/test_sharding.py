"""Splitting one query over ranks (imageproc_b200.sharding) on CPU with gloo
process groups: row bands of one score map with an (h - 1)-row halo, the
templates of a many-template bank split across ranks, and find_extremes of a
banded map through packed (value, index) keys. Each rank's share is scored by
the oracle here (the library on a GPU); the gathered results must equal the
one-rank results bit for bit, including first-occurrence ties
(src/template_matching.rs:490-507)."""

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from imageproc_b200 import sharding

ROOT = Path(__file__).resolve().parents[1]


def test_split_helpers():
    assert sharding.split_range(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert sharding.split_range(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]
    bands = sharding.band_rows(H=100, h=7, parts=3)  # 94 output rows
    assert [b[:2] for b in bands] == [(0, 32), (32, 63), (63, 94)]
    assert all(r1 - r0 == (y1 - y0) + 6 for y0, y1, r0, r1 in bands)


def test_packed_keys_first_occurrence():
    from oracle import oracle as O
    a = np.array([[3.0, 1.0, 5.0], [1.0, 5.0, 0.5], [0.5, 5.0, 1.0]], np.float32)
    keys = [sharding.band_extremes_keys(a[r:r + 1], r, 3) for r in range(3)]
    kmin = min(k[0] for k in keys)
    kmax = max(k[1] for k in keys)
    assert sharding.decode_extremes(kmin, kmax, 3) == O.find_extremes(a)
    assert sharding._from_i64(sharding._to_i64(kmin)) == kmin
    assert sharding._from_i64(sharding._to_i64((1 << 64) - 1)) == (1 << 64) - 1


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_band(image, template, method):
    from oracle import oracle as O
    return O.match_exact(image, template, method, None, precision=0, threads=1)


def _oracle_many(image, templates, method):
    from oracle import oracle as O
    return [O.find_extremes(O.match_exact(image, t, method, None, precision=0, threads=1)) for t in templates]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    from imageproc_b200 import sharding as S
    from imageproc_b200 import synthetic
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = {}
        image, template, _, _ = synthetic.blob_scene(W=160, H=97, tw=13, th=9, seed=21, n_blobs=12)
        for method in range(4):
            full, ext = S.match_template_bands(image, template, method, _oracle_band)
            out[("bands", method)] = (full, ext)
        # a periodic scene: every extreme is a tie across bands
        flat = np.tile(np.arange(10, dtype=np.uint8) * 20, (60, 12))
        full, ext = S.match_template_bands(flat, flat[:5, :7].copy(), 0, _oracle_band, gather_map=False)
        out[("ties", 0)] = (full, ext)
        image2, templates, _ = synthetic.value_noise_scene(W=128, H=96, n_templates=7, t=16, seed=8)
        out[("many", 3)] = S.match_templates_split(image2, templates, 3, _oracle_many)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_split_queries_equal_one_rank(world):
    import torch.multiprocessing as mp
    from imageproc_b200 import synthetic
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    image, template, _, _ = synthetic.blob_scene(W=160, H=97, tw=13, th=9, seed=21, n_blobs=12)
    flat = np.tile(np.arange(10, dtype=np.uint8) * 20, (60, 12))
    image2, templates, _ = synthetic.value_noise_scene(W=128, H=96, n_templates=7, t=16, seed=8)
    for rank in range(world):
        got = results[rank]
        for method in range(4):
            exp = O.match_exact(image, template, method, None, precision=0)
            full, ext = got[("bands", method)]
            assert np.array_equal(full.view(np.uint32), exp.view(np.uint32))
            assert ext == O.find_extremes(exp)
        _, ext = got[("ties", 0)]
        assert ext == O.find_extremes(O.match_exact(flat, flat[:5, :7].copy(), 0, None, precision=0))
        exp_many = [O.find_extremes(O.match_exact(image2, t, 3, None, precision=0)) for t in templates]
        assert got[("many", 3)] == exp_many
