"""The N > 1 plumbing of bench.py on CPU: world-size-2 gloo process groups.

The data path has no collective (each rank matches its own scene); what two
ranks share is the timing rule -- the max over ranks of each rank's device
time -- and the barriers around the timed region. These tests run that host
logic with the gloo backend, and launch the reference arm under torchrun with
two ranks, where only rank 0 may print its line.
"""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        # each rank's "device time"; the job's time is the slowest rank's
        got = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        bench.barrier(world)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    results = dict(q.get(timeout=5) for _ in range(2))
    assert results == {0: 15.0, 1: 15.0}


def test_ranks_match_independent_scenes():
    # weak scaling: rank r works on its own seeded scene (seed 1 + r)
    from imageproc_b200 import synthetic
    a = synthetic.blob_scene(W=256, H=128, tw=16, th=16, seed=1, n_blobs=8)
    b = synthetic.blob_scene(W=256, H=128, tw=16, th=16, seed=2, n_blobs=8)
    assert (a[0] != b[0]).any()


def test_reference_arm_under_torchrun_two_ranks():
    oracle_lib = ROOT / "oracle" / "_build" / "libtm_oracle.so"
    if not oracle_lib.exists():
        pytest.skip("oracle not built (python -c 'import __graft_entry__ as g; g.build()')")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--ref-step-s", "0.05"]
    env = dict(os.environ, OMP_NUM_THREADS="1", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port"
