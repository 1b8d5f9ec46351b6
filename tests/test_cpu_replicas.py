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
