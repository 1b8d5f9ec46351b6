"""Replica plumbing of bench.py --gpus N on CPU ranks (gloo, world size 2): the
barrier and the max over ranks of the per-rank step time."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from inching_b200 import replicas
    replicas.barrier()
    w, r = replicas.world()
    m = replicas.max_over_ranks(1.5 + r, device="cpu")
    q.put((r, w, m))
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 2.5), (1, 2, 2.5)]


def test_single_process_is_identity():
    from inching_b200 import replicas
    assert replicas.world() == (1, 0)
    assert replicas.max_over_ranks(3.25) == 3.25


def test_partition_by_size_balanced_and_complete():
    import numpy as np
    from inching_b200.batched import partition_by_size
    from inching_b200 import synth
    sizes = synth.batch_sizes(512, 300, 20000, seed=2)
    for W in (1, 2, 4, 8):
        parts = partition_by_size(sizes, W)
        allidx = sorted(i for p in parts for i in p)
        assert allidx == list(range(512))
        loads = [int(sizes[p].sum()) for p in parts]
        # greedy LPT: no rank exceeds the mean by more than the largest structure
        assert max(loads) - sum(loads) / W <= sizes.max()
        assert all(p == sorted(p) for p in parts)
    assert partition_by_size([5, 3], 4)[2:] == [[], []]


def _gather_rank(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from inching_b200.batched import gather_results, partition_by_size
    sizes = [30, 10, 20, 25, 5]
    mine = partition_by_size(sizes, world)[rank]
    local = {i: (np.full(3, float(i)), np.full((3, sizes[i], 3), float(i))) for i in mine}
    merged = gather_results(local)
    q.put((rank, None if merged is None else sorted((i, float(ev[0]), m.shape[1]) for i, (ev, m) in merged.items())))
    dist.destroy_process_group()


def test_sharded_batch_gather_gloo_world2():
    """The sharded batch's only exchange: rank 0 receives every structure's
    results, the other rank gets None."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[1] is None
    assert out[0] == [(0, 0.0, 30), (1, 1.0, 10), (2, 2.0, 20), (3, 3.0, 25), (4, 4.0, 5)]
