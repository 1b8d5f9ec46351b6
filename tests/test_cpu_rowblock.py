"""Row-block solver of one structure over several ranks, on CPU: the partition and
halo plan on real neighbour lists, and the distributed block solver on gloo
ranks (world sizes 1 and 3, so that a middle rank exchanges halos on both sides,
and 4 on a chain of globules whose ranks exchange with adjacent ranks only)
with dense row blocks of the oracle Hessian standing in for the GPU store rows.
Eigenvalues are checked against dense LAPACK, the gathered eigenvectors by their
residual and orthonormality."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import graph as og
from oracle import hessian as oh


def _structure(kind="globule"):
    """Atoms in reversed Cuthill-McKee order, their lists, and H + PlusI*I (dense).
    "globule": 400 atoms, a band nearly as wide as the structure; "chain": six
    touching 250-atom globules along x, whose band is narrow enough that each
    rank of four exchanges halos with its adjacent ranks only."""
    from inching_b200 import synth
    if kind == "globule":
        X = synth.globule(400, seed=5) / 10.0
    else:
        step = 2.0 * synth.globule_radius(250) * 0.95
        parts = []
        for i in range(6):
            g = synth.globule(250, seed=40 + i)
            parts.append(g - g.mean(axis=0) + np.array([i * step, 0.0, 0.0]))
        X = np.concatenate(parts) / 10.0
    deg, rp, cl = og.neighbor_lists(X, 8.0)
    order, _ = og.cuthill_mckee(rp, cl, deg)
    Xr = X[order]
    deg, rp, cl = og.neighbor_lists(Xr, 8.0)
    A, Ad = oh.hessian_lower(Xr, 8.0, 1.0)
    H = oh.full_from_lower(A, Ad).toarray()
    return Xr, rp, cl, H


class DenseRows:
    """Rows [a, b) of a dense H restricted to the columns of atoms [lo, hi), with
    the store's ext_matmul interface: the epilogue over every extended row, the
    halo rows without an H term."""

    def __init__(self, H, a, b, lo, hi):
        self.H64 = torch.from_numpy(np.ascontiguousarray(H[3 * a:3 * b, 3 * lo:3 * hi]))
        self.H32 = self.H64.float()
        self.own = slice(3 * (a - lo), 3 * (b - lo))

    def ext_matmul(self, X_ext, out, prec, alpha=1.0, gamma=0.0, beta=0.0, Yin=None, acc=None, mu=0.0):
        Y = torch.zeros_like(X_ext)
        Y[self.own] = (self.H64 if prec == 64 else self.H32) @ X_ext
        Y = alpha * Y + gamma * X_ext
        if Yin is not None and beta != 0.0:
            Y = Y + beta * Yin
        if acc is not None:
            acc += mu * Y
        out.copy_(Y)
        return out


def test_partition_halo_and_exchange_plan():
    from inching_b200.rowblock import exchange_plan, halo_ranges, row_partition
    _, rp, cl, H = _structure()
    n = len(rp) - 1
    for world in (1, 2, 3, 5):
        parts = row_partition(rp, world)
        assert parts[0][0] == 0 and parts[-1][1] == n
        assert all(p[1] == q[0] for p, q in zip(parts, parts[1:])) and all(a < b for a, b in parts)
        work = [(rp[b] - rp[a]) + (b - a) for a, b in parts]
        assert max(work) <= 1.5 * sum(work) / world
        ranges = halo_ranges(rp, cl, parts)
        for (a, b), (lo, hi) in zip(parts, ranges):
            assert lo <= a < b <= hi
            rows = H[3 * a:3 * b]
            assert not rows[:, :3 * lo].any() and not rows[:, 3 * hi:].any()   # the halo holds every column
        plans = [exchange_plan(parts, ranges, r) for r in range(world)]
        for r in range(world):
            sends, recvs = plans[r]
            for peer, u, v in sends:               # what r sends, peer expects from r
                assert (r, u, v) in plans[peer][1]
            got = sorted((u, v) for _, u, v in recvs)
            lo, hi = ranges[r]
            a, b = parts[r]
            need = [(u, v) for u, v in ((lo, a), (b, hi)) if u < v]
            # the received pieces tile the two halo slabs exactly
            cover = set()
            for u, v in got:
                cover.update(range(u, v))
            assert cover == set().union(*[set(range(u, v)) for u, v in need]) if need else not cover
    with pytest.raises(AssertionError):
        row_partition(rp, n + 1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _solve(world_rank, world, port, q, kind="globule"):
    import torch.distributed as dist
    from inching_b200.rowblock import (RowBlockComm, RowBlockOperator, chfsi_rowblock, gather_rows, halo_ranges,
                                       row_partition)
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=world_rank, world_size=world)
    torch.set_num_threads(1)
    Xr, rp, cl, H = _structure(kind)
    comm = RowBlockComm()
    parts = row_partition(rp, comm.world)
    ranges = halo_ranges(rp, cl, parts)
    a, b = parts[comm.rank]
    lo, hi = ranges[comm.rank]
    A = RowBlockOperator(DenseRows(H, a, b, lo, hi), parts, ranges, comm, Xr.shape[0], torch.device("cpu"))
    Q = torch.from_numpy(oh.rigid_body_basis(Xr))[:, 3 * a:3 * b].contiguous()
    out = {}
    for precision, tol in (("f64", 1e-9), ("mixed", 1e-6)):
        ev, V, info = chfsi_rowblock(A, 20, tol=tol, Q=Q, precision=precision, return_info=True)
        full = gather_rows(comm, V, parts)
        out[precision] = (ev.numpy(), None if full is None else full.numpy(), info["converged"],
                          info["max_rel_residual"], info["halo_bytes"])
    if world > 1:
        dist.destroy_process_group()
    q.put((comm.rank, out))


def _check(results, kind="globule"):
    _, _, _, H = _structure(kind)
    w = np.linalg.eigvalsh(H)
    for precision, tol in (("f64", 1e-9), ("mixed", 1e-6)):
        evs = [r[precision][0] for r in results]
        for ev in evs[1:]:
            assert np.array_equal(ev, evs[0])      # every rank reports the same eigenvalues
        ev, V, conv, res, _ = results[0][precision]
        assert conv and res <= 1.5 * tol
        assert np.max(np.abs(ev - w[6:26]) / w[6:26]) < (1e-10 if precision == "f64" else 1e-5)
        assert np.abs(V.T @ V - np.eye(20)).max() < 1e-10
        R = H @ V - V * ev[None, :]
        assert np.linalg.norm(R, axis=0).max() <= 1.5 * tol * 1.03 * w[-1]
    if len(results) > 1:
        assert all(r["f64"][4] > 0 for r in results)   # halos were exchanged


def test_rowblock_solver_single_rank():
    class Q:
        def __init__(self):
            self.items = []

        def put(self, x):
            self.items.append(x)

    q = Q()
    _solve(0, 1, 0, q)
    _check([q.items[0][1]])


def test_rowblock_solver_gloo_world3():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_solve, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1]["f64"][1] is None and got[2]["f64"][1] is None    # gathered on rank 0 only
    _check([got[0], got[1], got[2]])


def test_rowblock_solver_gloo_world4_chain():
    from inching_b200.rowblock import exchange_plan, halo_ranges, row_partition
    _, rp, cl, _ = _structure("chain")
    parts = row_partition(rp, 4)
    ranges = halo_ranges(rp, cl, parts)
    for r in range(4):
        sends, recvs = exchange_plan(parts, ranges, r)
        assert {p for p, _, _ in sends} | {p for p, _, _ in recvs} <= {r - 1, r + 1}
        assert recvs and 0 < ranges[r][1] - ranges[r][0] < len(rp) - 1     # partial halos
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_solve, args=(r, 4, port, q, "chain")) for r in range(4)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    _check([got[r] for r in range(4)], "chain")
