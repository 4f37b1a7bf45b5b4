"""Multi-rank logic of bench.py on CPU: world size 2 over gloo.

Each rank advances its own seeded ensemble (no data-path collective); the
whole-job figure is all ranks' lattice updates over the slowest rank's
time.  This checks the sharding and the two reductions the bench uses.
"""
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    from uq_b200 import workloads as W

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        samples = W.uq_ensemble(n=8, seed=bench.rank_seed(1234, rank))
        nodes = sum(d["nx"] * d["ny"] for d in samples)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        total = bench.reduce_over_ranks(nodes, dist, "sum", "cpu")
        slowest = bench.reduce_over_ranks(ms, dist, "max", "cpu")
        out[rank] = dict(nodes=nodes, total=total, slowest=slowest,
                         value=bench.aggregate_mlups(total, 50, slowest),
                         sides=[d["nx"] for d in samples])
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    r0, r1 = res[0], res[1]
    assert r0["sides"] != r1["sides"]  # ranks hold different shards
    assert r0["total"] == r1["total"] == r0["nodes"] + r1["nodes"]
    assert r0["slowest"] == r1["slowest"] == 15.0
    assert r0["value"] == pytest.approx((r0["nodes"] + r1["nodes"]) * 50 / 15e3)


def test_rank_zero_is_the_single_gpu_run():
    import sys

    sys.path.insert(0, ROOT)
    import bench
    from uq_b200 import workloads as W

    assert bench.rank_seed(1234, 0) == 1234
    assert bench.reduce_over_ranks(7.0, None, "max", "cpu") == 7.0
    one = W.uq_ensemble(n=8, seed=1234)
    assert [d["nx"] for d in one] == [d["nx"] for d in W.uq_ensemble(n=8, seed=bench.rank_seed(1234, 0))]
