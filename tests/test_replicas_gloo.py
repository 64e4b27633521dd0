"""The multi-GPU path on the host: two gloo ranks exercise the replica
bookkeeping that bench.py uses under torchrun (max of the ranks' times, sums
of per-rank counts, the split of independent instances), and a non-zero rank
of the reference arm leaves without work.  No GPU is involved.
"""
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    from datetime import timedelta

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from pywignercuda2_b200 import replicas
        info = replicas.rank_info()
        mx = replicas.max_over_ranks(1.5 + rank)
        sm = replicas.sum_over_ranks(10 * (rank + 1))
        replicas.barrier()
        mine = replicas.shard(range(48), rank, world)
        q.put((rank, info, mx, sm, mine))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, info, mx, sm, mine in out:
        assert info == (2, rank, rank)
        assert mx == 2.5            # the slowest rank's time
        assert sm == 30             # 10 + 20
        assert len(mine) == 24
    assert sorted(out[0][4] + out[1][4]) == list(range(48))


def test_shard_single_rank():
    sys.path.insert(0, ROOT)
    from pywignercuda2_b200 import replicas
    assert replicas.shard(range(5), 0, 1) == [0, 1, 2, 3, 4]
    assert replicas.max_over_ranks(3.0) == 3.0    # no process group: the value itself


def test_reference_arm_nonzero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
