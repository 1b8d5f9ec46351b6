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

from .deflation import rigid_body_basis
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


def batched_normal_modes(structs, k=32, *, units="nm", rc_gamma_A=8.0, plus_i=1.0, tol=1e-6, precision="mixed",
                         degree=24, bucket_ratio=1.6, seed=0, verbose=False):
    t0 = time.perf_counter()
    structs = [np.asarray(X, dtype=np.float64) / (10.0 if units == "A" else 1.0) for X in structs]
    sizes = np.array([X.shape[0] for X in structs])
    results = [None] * len(structs)
    infos = []
    rc = rc_gamma_A / 10.0
    for bucket in buckets_by_size(sizes, bucket_ratio):
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
        Qp = torch.zeros((len(bucket), 6, n_max), dtype=torch.float64, device=Xd.device)
        for t in range(len(bucket)):
            a0, a1 = int(atom_off[t]), int(atom_off[t + 1])
            Qp[t, :, :3 * (a1 - a0)] = rigid_body_basis(Xd[a0:a1])
        ev, V, info = chfsi_batched(H, 3 * atom_off, k, tol=tol, Qp=Qp, precision=precision, degree=degree,
                                    seed=seed, verbose=verbose)
        ev = ev.cpu().numpy()
        for t, i in enumerate(bucket):
            a0, a1 = int(atom_off[t]), int(atom_off[t + 1])
            modes = V[3 * a0:3 * a1].t().reshape(k, a1 - a0, 3)
            results[i] = (ev[t] - plus_i, modes)
        info = dict(info)
        info.update(n_atoms=int(atom_off[-1]), sizes=(int(sizes[bucket].min()), int(sizes[bucket].max())))
        infos.append(info)
    torch.cuda.synchronize()
    return results, dict(buckets=infos, seconds=time.perf_counter() - t0, structures=len(structs))
