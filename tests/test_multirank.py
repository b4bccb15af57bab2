"""bench.py's multi-rank host logic on CPU: two gloo ranks (world_size 2)
take the max of the per-rank times and the sum of the per-rank work, the
replicas draw distinct seeded workloads, and the reference arm runs on
rank 0 only.  No GPU."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist

    w, r, _ = bench.dist_setup()
    try:
        assert dist.get_backend() == "gloo"
        mx = bench.reduce_max(10.0 + r, w)
        sm = bench.reduce_sum(100.0 * (r + 1), w)
        bench.barrier(w)
        lat, wts, src = bench.make_workload(bench.SEED + 7919 * r, 12, 10, 2, 4)
        args = type("A", (), dict(nx=12, ny=10, nz=2, sources=2, steps=1, warmup=0))()
        ref = bench.run_reference(args, w, r, r)
        q.put((r, mx, sm, src.tolist(), float(wts[:64].sum()), ref is None))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_reduce_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, *rest = q.get(timeout=240)
        out[r] = rest
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert out[r][0] == 11.0  # max over ranks of the per-rank time
        assert out[r][1] == 300.0  # sum over ranks of the per-rank work
    assert out[0][2] != out[1][2] or out[0][3] != out[1][3]  # distinct replica workloads
    assert out[0][4] is False and out[1][4] is True  # reference arm: rank 0 only
