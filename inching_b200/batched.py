"""Normal modes of many independent structures in one batched solve.

Structures are sorted by size and grouped into buckets whose sizes differ by at
most a factor `bucket_ratio`; each bucket is laid out on a lattice (no neighbour
pair can cross structures, which is checked), assembled into one block-diagonal
Hessian store and solved by `solvers.batched.chfsi_batched`: every Chebyshev
step of a bucket is one SpMM launch for all its structures.  Atoms keep their
input order inside each structure (the ordering only affects locality, not the
modes).  Returns, per structure and in input order, eigenvalues with PlusI
removed and eigenvectors shaped (k, N_s, 3) -- the reference drivers' layout.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from .deflation import rigid_body_basis_padded
from .hessian import HessianStore
from .solvers.batched import chfsi_batched


def buckets_by_size(sizes, ratio=1.6, max_atoms=4_000_000):
    order = np.argsort(sizes, kind="stable")
    out, cur = [], []
    for i in order:
        if cur and (sizes[i] > ratio * sizes[cur[0]] or sum(sizes[c] for c in cur) + sizes[i] > max_atoms):
            out.append(cur)
            cur = []
        cur.append(int(i))
    if cur:
        out.append(cur)
    return out


def lattice_layout(structs_nm, rc_nm):
    """Centre each structure and place it on a cubic lattice whose spacing exceeds
    the largest diameter plus twice the cutoff."""
    cents = [X - X.mean(axis=0) for X in structs_nm]
    rad = max(float(np.sqrt((c ** 2).sum(axis=1)).max()) for c in cents)
    spacing = 2.0 * rad + 2.0 * rc_nm + 0.5
    side = int(np.ceil(len(cents) ** (1.0 / 3.0)))
    parts = []
    for t, c in enumerate(cents):
        ix, iy, iz = t % side, (t // side) % side, t // (side * side)
        parts.append(c + spacing * np.array([ix, iy, iz], dtype=np.float64))
    return np.concatenate(parts, axis=0)


def _bucket_warm_start(Xd, sid, n_struct, k, guard, seed, bead_edge_A=6.0, rc_bead_A=12.0):
    """Per-structure bead models of a laid-out bucket, solved together (their bead
    Hessian is block-diagonal too), prolonged to the atoms: (3N, m) FP64."""
    edge = bead_edge_A / 10.0
    lo = Xd.min(dim=0).values
    c = torch.floor((Xd - lo) / edge).long()
    dims = c.max(dim=0).values + 1
    key = ((sid * dims[0] + c[:, 0]) * dims[1] + c[:, 1]) * dims[2] + c[:, 2]
    uniq, bead = torch.unique(key, return_inverse=True)       # sorted: beads grouped by structure
    nb = uniq.shape[0]
    one = torch.ones_like(bead, dtype=torch.float64)
    cnt = torch.zeros(nb, dtype=torch.float64, device=Xd.device).index_add_(0, bead, one)
    pos = torch.zeros((nb, 3), dtype=torch.float64, device=Xd.device).index_add_(0, bead, Xd) / cnt[:, None]
    bead_sid = torch.zeros(nb, dtype=torch.long, device=Xd.device).index_copy_(0, bead, sid)
    nbs = torch.bincount(bead_sid, minlength=n_struct).cpu().numpy()
    boff = np.concatenate([[0], np.cumsum(nbs)])
    Hb = HessianStore(pos, rc_bead_A, plus_i=1.0)
    m = int(min(k + guard, 3 * nbs.min() - 7))
    Qb = rigid_body_basis_padded(pos, boff, int(3 * nbs.max()))
    _, Vb, _ = chfsi_batched(Hb, 3 * boff, m - 2, tol=1e-3, Qp=Qb, precision="mixed", guard=2, seed=seed + 7)
    return Vb.reshape(nb, 3, -1).index_select(0, bead).reshape(3 * Xd.shape[0], -1)


def batched_normal_modes(structs, k=32, *, units="nm", rc_gamma_A=8.0, plus_i=1.0, tol=1e-6, precision="mixed",
                         degree=24, bucket_ratio=1.6, seed=0, verbose=False, profile=False, warm_start=None,
                         guard=None):
    t0 = time.perf_counter()
    structs = [np.asarray(X, dtype=np.float64) / (10.0 if units == "A" else 1.0) for X in structs]
    if not structs:
        return [], dict(buckets=[], seconds=0.0, structures=0)
    sizes = np.array([X.shape[0] for X in structs])
    results = [None] * len(structs)
    infos = []
    rc = rc_gamma_A / 10.0
    import time as _t
    for bucket in buckets_by_size(sizes, bucket_ratio):
        tb0 = _t.perf_counter()
        Xcat = lattice_layout([structs[i] for i in bucket], rc)
        Xd = torch.from_numpy(Xcat).cuda()
        precisions = ("f64", "f32") if precision == "mixed" else ("f64",)
        H = HessianStore(Xd, rc_gamma_A, plus_i=plus_i, precisions=precisions)
        atom_off = np.concatenate([[0], np.cumsum(sizes[bucket])])
        # block-diagonal check: every neighbour pair stays inside one structure
        sid = torch.repeat_interleave(torch.arange(len(bucket), device=Xd.device),
                                      torch.from_numpy(sizes[bucket]).to(Xd.device))
        rows = torch.repeat_interleave(sid, H.degree.long())
        if not bool((sid[H.cols.long()] == rows).all()):
            raise AssertionError("ABORTED. structures overlap in the batched layout")
        n_max = int(3 * sizes[bucket].max())
        Qp = rigid_body_basis_padded(Xd, atom_off, n_max)
        Y0 = None
        if warm_start == "coarse":
            guard = max(16, int(np.ceil(0.5 * k)))
            Y0 = _bucket_warm_start(Xd, sid, len(bucket), k, guard, seed)
        if profile:
            torch.cuda.synchronize()
        tb1 = _t.perf_counter()
        ev, V, info = chfsi_batched(H, 3 * atom_off, k, tol=tol, Qp=Qp, precision=precision, degree=degree,
                                    seed=seed, verbose=verbose, profile=profile, Y0=Y0, guard=guard)
        if profile:
            torch.cuda.synchronize()
        tb2 = _t.perf_counter()
        ev = ev.cpu().numpy()
        for t, i in enumerate(bucket):
            a0, a1 = int(atom_off[t]), int(atom_off[t + 1])
            modes = V[3 * a0:3 * a1].t().reshape(k, a1 - a0, 3)
            results[i] = (ev[t] - plus_i, modes)
        info = dict(info)
        info.update(n_atoms=int(atom_off[-1]), sizes=(int(sizes[bucket].min()), int(sizes[bucket].max())),
                    setup_s=round(tb1 - tb0, 3), solve_s=round(tb2 - tb1, 3))
        infos.append(info)
    torch.cuda.synchronize()
    return results, dict(buckets=infos, seconds=time.perf_counter() - t0, structures=len(structs))


# ---------------------------------------------------------------------------
# Several GPUs: the structures are independent, so the batch shards with no
# data-path collective (one process per GPU, torch.distributed for the plumbing).
# ---------------------------------------------------------------------------
def partition_by_size(sizes, world_size):
    """Greedy size-balanced partition: structures in decreasing size, each to the
    rank with the fewest atoms so far.  Returns one ascending index list per rank."""
    sizes = np.asarray(sizes)
    load = np.zeros(world_size, dtype=np.int64)
    parts = [[] for _ in range(world_size)]
    for i in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def gather_results(local, dst=0):
    """Collect every rank's {structure index: (eigenvalues, modes)} (host arrays) on
    rank dst; the final and only exchange of the sharded batch.  Other ranks get None."""
    import torch.distributed as dist
    from .replicas import world
    W, R = world()
    if W == 1:
        return dict(local)
    out = [None] * W if R == dst else None
    dist.gather_object(list(local.items()), out, dst=dst)
    if R != dst:
        return None
    merged = {}
    for part in out:
        merged.update(dict(part))
    return merged


def sharded_batched_normal_modes(structs, k=32, *, gather=True, **kw):
    """batched_normal_modes over this rank's share of `structs` (partition_by_size
    over the ranks of the default process group; a single process takes all).
    Returns ({index: (eigenvalues, modes)} -- every structure's, as host arrays, on
    rank 0 after the gather; this rank's, modes on the device, without it -- and
    this rank's info with its indices)."""
    from .replicas import world
    W, R = world()
    sizes = [np.asarray(X).shape[0] for X in structs]
    mine = partition_by_size(sizes, W)[R]
    res, info = batched_normal_modes([structs[i] for i in mine], k, **kw)
    info = dict(info, indices=mine, rank=R, world=W, atoms=int(sum(sizes[i] for i in mine)))
    local = {i: r for i, r in zip(mine, res)}
    if not gather:
        return local, info
    host = {i: (ev, m.cpu().numpy()) for i, (ev, m) in local.items()}
    return gather_results(host), info
