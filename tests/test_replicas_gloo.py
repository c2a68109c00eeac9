"""Multi-process host logic of `bench.py --gpus N` on CPU (gloo, world size 2): one process per
rank, each with its own replica seed; the timed interval is the maximum over ranks and the
whole-job rate counts every rank's atoms.  The GPU path uses the same functions over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_ms = 10.0 + 5.0 * rank
    mx = bench.max_over_ranks(local_ms, dist, torch.device("cpu"))
    dist.barrier()
    q.put((rank, mx, bench.aggregate_rate(world, 1000, 10, mx)))
    dist.destroy_process_group()


def test_max_over_ranks_and_rate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]          # the slower rank's time on every rank
    assert res[0][2] == pytest.approx(2 * 1000 * 10 / 0.015)


def test_partition_replicas_by_atom_count():
    """The 512-replica batch split over 2, 4 and 8 ranks: every replica exactly once, loads within
    one (largest) replica of each other, deterministic."""
    import sys
    import numpy as np
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from copy_gpu_b200 import systems
    r = systems.replicas(n_rep=512, seed=11)
    sizes = np.diff(r["offsets"])
    for world in (1, 2, 4, 8):
        parts = bench.partition_replicas(sizes, world)
        assert sorted(k for p in parts for k in p) == list(range(512))
        loads = [int(sizes[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= sizes.max()
        assert parts == bench.partition_replicas(sizes, world)
        sub, boxes, offs = bench.replica_subset(r, [None] * 512, parts[0])
        assert offs[-1] == loads[0] == sub["pos"].shape[0] and len(boxes) == len(parts[0])
        k = parts[0][-1]
        assert np.array_equal(sub["pos"][offs[-2]:offs[-1]], r["pos"][r["offsets"][k]:r["offsets"][k + 1]])
