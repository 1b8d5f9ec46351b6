"""One structure on several GPUs: the block eigensolver over a 1-D row-block
partition of the Hessian in Cuthill-McKee order (no reference counterpart: the
reference solves a structure on one GPU).

Layout.  Rank r owns the contiguous atom range [a_r, b_r) of the reordered
structure: its rows of the store, and the same rows of every block vector
(dof rows [3 a_r, 3 b_r)).  Its store rows are built from the neighbour lists
with the columns rebased to the extended range [lo_r, hi_r), the smallest atom
range that holds every column of those rows.  Cuthill-McKee keeps that range a
band around [a_r, b_r), so the halo rows [lo_r, a_r) and [b_r, hi_r) are two
contiguous slabs owned by the neighbouring ranks.

Communication.
  * one halo exchange per SpMM: every rank sends each peer the rows of its own
    range that fall in the peer's halo, as point-to-point messages (NCCL send /
    recv over NVLink between GPUs; gloo on CPU);
  * every inner product of the block solver (Gram matrices of Cholesky-QR,
    projections against the rigid-body basis and the locked modes, the
    Rayleigh-Ritz matrix, residual norms, Lanczos dot products) is a local GEMM
    followed by one FP64 all-reduce of a small matrix;
  * the small eigenproblems are solved on rank 0 and broadcast, so that every
    rank takes the same locking decisions.

The per-rank work is the single-GPU solver's with the matrix and the block cut
by rows, and the results equal the single-GPU solver's to the solver tolerance
(the random start differs).  The Chebyshev filter keeps its two recurrence
buffers at the size of the extended range, so the recurrence's epilogue
(alpha H X + gamma X + beta Yin) stays fused in the SpMM as on one GPU.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

from .solvers.chfsi import STALL_RESTART, default_guard


# ---------------------------------------------------------------------------
# Partition and halo plan (pure host logic, identical on every rank)
# ---------------------------------------------------------------------------
def row_partition(rowptr, world):
    """Contiguous atom ranges [(a, b)] for `world` ranks, cut where the running
    count of (stored entries + rows) crosses r / world of the total: the SpMM's
    work per rank is about equal.  Every range holds at least one atom."""
    rp = np.asarray(rowptr.cpu() if torch.is_tensor(rowptr) else rowptr, dtype=np.int64)
    n = rp.shape[0] - 1
    if not 1 <= world <= n:
        raise AssertionError(f"ABORTED. cannot cut {n} atoms into {world} row blocks")
    work = rp + np.arange(n + 1)                  # entries + rows before each atom
    cuts = [0]
    for r in range(1, world):
        c = int(np.searchsorted(work, work[-1] * r / world))
        cuts.append(min(max(c, cuts[-1] + 1), n - (world - r)))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def halo_ranges(rowptr, cols, parts):
    """[(lo, hi)] per range: the smallest atom range holding [a, b) and every
    column of rows a..b-1.  The column minima and maxima are taken where cols
    lives (a device tensor stays on the device)."""
    rp = np.asarray(rowptr.cpu() if torch.is_tensor(rowptr) else rowptr, dtype=np.int64)
    out = []
    for a, b in parts:
        seg = cols[int(rp[a]):int(rp[b])]
        if len(seg):
            out.append((min(a, int(seg.min())), max(b, int(seg.max()) + 1)))
        else:
            out.append((a, b))
    return out


def exchange_plan(parts, ranges, rank):
    """(sends, recvs) of `rank`: lists of (peer, u, v), atom rows [u, v).  A rank
    sends a peer the part of its own range that lies in the peer's halo, and
    receives from each peer the part of the peer's range in its own halo."""
    def pieces(own, need):
        a, b = own
        lo, hi, na, nb = need
        got = []
        for u, v in ((lo, na), (nb, hi)):           # the two halo slabs
            s, e = max(a, u), min(b, v)
            if s < e:
                got.append((s, e))
        return got

    sends, recvs = [], []
    a_me, b_me = parts[rank]
    lo_me, hi_me = ranges[rank]
    for peer in range(len(parts)):
        if peer == rank:
            continue
        a_p, b_p = parts[peer]
        lo_p, hi_p = ranges[peer]
        sends += [(peer, u, v) for u, v in pieces((a_me, b_me), (lo_p, hi_p, a_p, b_p))]
        recvs += [(peer, u, v) for u, v in pieces((a_p, b_p), (lo_me, hi_me, a_me, b_me))]
    return sends, recvs


# ---------------------------------------------------------------------------
# Communicator
# ---------------------------------------------------------------------------
class RowBlockComm:
    """The collectives the row-block solver uses, over a torch.distributed group
    (NCCL for CUDA tensors, gloo for CPU tensors), or local no-ops when
    torch.distributed is not initialised (one rank)."""

    def __init__(self, group=None):
        self.group = group
        self.on = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if self.on else 0
        self.world = dist.get_world_size(group) if self.on else 1

    def allreduce_(self, t):
        if self.on and self.world > 1:
            dist.all_reduce(t, group=self.group)
        return t

    def broadcast_(self, t, src=0):
        if self.on and self.world > 1:
            dist.broadcast(t, src=self._global(src), group=self.group)
        return t

    def _global(self, r):
        return dist.get_global_rank(self.group, r) if self.group is not None else r

    def p2p(self, sends, recvs):
        """sends / recvs: lists of (peer, tensor); all posted at once, then waited."""
        if not (sends or recvs):
            return
        ops = [dist.P2POp(dist.isend, t, self._global(p), self.group) for p, t in sends]
        ops += [dist.P2POp(dist.irecv, t, self._global(p), self.group) for p, t in recvs]
        for w in dist.batch_isend_irecv(ops):
            w.wait()


# ---------------------------------------------------------------------------
# Operator: halo exchange + local rows of H
# ---------------------------------------------------------------------------
class StoreRows:
    """Rows [a, b) of the Hessian store with columns rebased to [lo, hi), built by
    the package's neighbour lists and assembly kernels: a store over the atoms
    [lo, hi) whose halo atoms have no entries, so a product's halo rows carry no
    H term (callers overwrite or drop them)."""

    def __init__(self, X_nm, rc_gamma_A, plus_i, rowptr, cols, a, b, lo, hi, precisions=("f64", "f32")):
        from .hessian import HessianStore
        dev = X_nm.device
        e0, e1 = int(rowptr[a]), int(rowptr[b])
        counts = torch.zeros(hi - lo, dtype=torch.int64, device=dev)
        counts[a - lo:b - lo] = rowptr[a + 1:b + 1] - rowptr[a:b]
        rp = torch.zeros(hi - lo + 1, dtype=torch.int64, device=dev)
        rp[1:] = torch.cumsum(counts, 0)
        cl = (cols[e0:e1] - lo).to(torch.int32).contiguous()
        deg = counts.to(torch.int32)
        self.store = HessianStore(X_nm[lo:hi].contiguous(), rc_gamma_A, plus_i=plus_i, precisions=precisions,
                                  graph_=(deg, rp, cl))
        self.own = slice(3 * (a - lo), 3 * (b - lo))
        self.nnz_blocks = e1 - e0

    def ext_matmul(self, X_ext, out, prec, **epilogue):
        """out = alpha H_rows X_ext + gamma X_ext + beta Yin (+ acc) over all rows of
        the extended range, in one fused SpMM (the single-GPU store's epilogue)."""
        return self.store.matmul(X_ext, out=out, prec=prec, **epilogue)

    def local_matmul(self, X_ext, prec):
        """This rank's rows of H X_ext."""
        return self.store.matmul(X_ext, prec=prec)[self.own]


@dataclass
class _Layout:
    parts: list
    ranges: list
    rank: int

    @property
    def a(self):
        return self.parts[self.rank][0]

    @property
    def b(self):
        return self.parts[self.rank][1]

    @property
    def lo(self):
        return self.ranges[self.rank][0]

    @property
    def hi(self):
        return self.ranges[self.rank][1]


class RowBlockOperator:
    """H applied to row-distributed blocks: `matmul` takes this rank's rows of X
    (3 (b - a), w) and returns its rows of alpha H X + gamma X + beta Yin (+ acc),
    the interface of the single-GPU store, after one halo exchange.

    local: object with ext_matmul(X_ext, out, prec, alpha=, gamma=, beta=, Yin=)
    computing alpha H_rows X_ext + gamma X_ext + beta Yin over every row of the
    extended range [lo, hi) (StoreRows; the halo rows have no H term)."""

    def __init__(self, local, parts, ranges, comm: RowBlockComm, n_atoms, device):
        self.local = local
        self.comm = comm
        self.lay = _Layout(list(parts), list(ranges), comm.rank)
        if len(parts) != comm.world:
            raise AssertionError(f"ABORTED. {len(parts)} row blocks for {comm.world} ranks")
        self.n_atoms = int(n_atoms)
        self.shape = (3 * self.n_atoms, 3 * self.n_atoms)
        self.ndim = 2
        self.device = device
        self.n_local = 3 * (self.lay.b - self.lay.a)
        self.sends, self.recvs = exchange_plan(self.lay.parts, self.lay.ranges, comm.rank)
        self.n_spmm = 0
        self.halo_bytes = 0
        # all ranks check the partition together before any point-to-point message
        tot = torch.tensor([float(self.n_local)], dtype=torch.float64, device=device)
        if int(comm.allreduce_(tot).item()) != self.shape[0]:
            raise AssertionError("ABORTED. the row blocks do not cover the structure")

    @property
    def n_ext(self):
        """Dof rows of the extended range [lo, hi)."""
        return 3 * (self.lay.hi - self.lay.lo)

    @property
    def own(self):
        """This rank's rows within the extended range."""
        off = 3 * (self.lay.a - self.lay.lo)
        return slice(off, off + self.n_local)

    def exchange_(self, Xe):
        """Refresh the halo rows of an extended block Xe (3 (hi - lo), w) in place
        from the peers' own rows; Xe's own rows are sent to the peers that need
        them.  Every message is a contiguous row slab of Xe."""
        lay = self.lay
        snd = [(p, Xe[3 * (u - lay.lo):3 * (v - lay.lo)]) for p, u, v in self.sends]
        rcv = [(p, Xe[3 * (u - lay.lo):3 * (v - lay.lo)]) for p, u, v in self.recvs]
        self.comm.p2p(snd, rcv)
        self.halo_bytes += sum(t.numel() * t.element_size() for _, t in rcv)
        return Xe

    def matmul(self, X, out=None, prec=None, alpha=1.0, gamma=0.0, beta=0.0, Yin=None, acc=None, mu=0.0, **kw):
        if kw.get("Q") is not None:
            raise AssertionError("ABORTED. the row-block operator deflates by projection, not by a Hotelling term")
        if prec is None:
            prec = 64 if X.dtype == torch.float64 else 32
        Xe = torch.empty((self.n_ext,) + tuple(X.shape[1:]), dtype=X.dtype, device=X.device)
        Xe[self.own] = X
        Ye = torch.empty_like(Xe)
        self.local.ext_matmul(self.exchange_(Xe), Ye, prec)
        Y = Ye[self.own]
        self.n_spmm += 1
        if alpha != 1.0:
            Y = Y * alpha
        if gamma != 0.0:
            Y = Y + gamma * X
        if Yin is not None and beta != 0.0:
            Y = Y + beta * Yin
        if acc is not None:
            acc += mu * Y
        if out is None:
            return Y
        out.copy_(Y)
        return out


class _RowFilter:
    """The scaled Chebyshev filter of solvers.chfsi._Filter on extended blocks:
    the recurrence's two buffers hold the atoms [lo, hi); before each product the
    halo rows of the vector being multiplied are refreshed from the peers, and
    the recurrence's epilogue (alpha, gamma, beta Yin) runs inside the local
    SpMM over all extended rows.  A result's halo rows (no H term) are
    overwritten by the next exchange before any product reads them, and the
    epilogue is row-local, so the own rows are exact."""

    def __init__(self, A: "RowBlockOperator", prec):
        self.A = A
        self.prec = prec
        self.n_spmm = 0

    def __call__(self, X64, m, a, b, a0):
        A = self.A
        dt = torch.float64 if self.prec == 64 else torch.float32
        e = (b - a) / 2.0
        c = (b + a) / 2.0
        sigma = e / (a0 - c)
        sigma1 = sigma
        tau = 2.0 / sigma1
        w = X64.shape[1]
        wp = (w + 7) // 8 * 8          # aligned width for the vector-gather SpMM
        X = torch.zeros((A.n_ext, wp), dtype=dt, device=X64.device)
        X[A.own, :w] = X64
        Y = torch.empty_like(X)
        A.local.ext_matmul(A.exchange_(X), Y, self.prec, alpha=sigma1 / e, gamma=-sigma1 * c / e)
        self.n_spmm += 1
        for _ in range(2, m + 1):
            s2 = 1.0 / (tau - sigma)
            # X <- 2 s2/e (H Y - c Y) - sigma s2 X, written over X, then swap
            A.local.ext_matmul(A.exchange_(Y), X, self.prec, alpha=2.0 * s2 / e, gamma=-2.0 * s2 * c / e,
                               beta=-sigma * s2, Yin=X)
            X, Y = Y, X
            sigma = s2
            self.n_spmm += 1
        A.n_spmm += self.n_spmm
        return Y[A.own, :w].to(torch.float64)


# ---------------------------------------------------------------------------
# Distributed building blocks of the block solver
# ---------------------------------------------------------------------------
def _gram(comm, A, B):
    return comm.allreduce_((A.t() @ B).contiguous())


def _colnorms(comm, R):
    return torch.sqrt(comm.allreduce_((R * R).sum(dim=0).contiguous()))


def _project_out(comm, Y, B):
    """Y <- Y - B^T (B Y) for rows B (r, n_local) of a globally orthonormal basis, twice."""
    if B is None or B.shape[0] == 0:
        return Y
    for _ in range(2):
        Y = Y - B.t() @ comm.allreduce_((B @ Y).contiguous())
    return Y


def _cholqr(comm, Y, n_global):
    """Cholesky-QR twice on the global Gram matrix.  A Gram matrix that is not
    numerically positive gets one shifted pass first (shift 11 (m p + p (p+1)) u
    ||G||, Fukaya et al., SIAM J. Sci. Comput. 42 (2020), shifted CholeskyQR3)."""
    p = Y.shape[1]
    shifted = False
    passes = 0
    while passes < 2:
        G = _gram(comm, Y, Y)
        R, info = torch.linalg.cholesky_ex(G, upper=True)
        if int(info) != 0:
            if shifted:
                raise AssertionError("ABORTED. the block lost rank (shifted Cholesky-QR failed)")
            s = 11.0 * (n_global * p + p * (p + 1)) * float(torch.finfo(torch.float64).eps) * float(G.diagonal().sum())
            R, info = torch.linalg.cholesky_ex(G + s * torch.eye(p, dtype=G.dtype, device=G.device), upper=True)
            shifted = True
            if int(info) != 0:
                raise AssertionError("ABORTED. the block lost rank (shifted Cholesky-QR failed)")
        else:
            passes += 1
        Rinv = torch.linalg.solve_triangular(R, torch.eye(p, dtype=R.dtype, device=R.device), upper=True)
        Y = Y @ Rinv
    return Y


def _eigh_bcast(comm, G):
    """Eigenpairs of the symmetric G, solved on rank 0 and broadcast."""
    p = G.shape[0]
    buf = torch.empty((p + 1, p), dtype=torch.float64, device=G.device)
    if comm.rank == 0:
        th, W = torch.linalg.eigh(0.5 * (G + G.t()))
        buf[0] = th
        buf[1:] = W
    comm.broadcast_(buf, 0)
    return buf[0].cpu().numpy(), buf[1:]


def _rr(comm, A, Y, prec):
    if prec == 64:
        HY = A.matmul(Y.contiguous(), prec=64)
    else:
        HY = A.matmul(Y.to(torch.float32).contiguous(), prec=32).to(torch.float64)
    th, W = _eigh_bcast(comm, _gram(comm, Y, HY))
    return th, Y @ W, HY @ W


def spectrum_bound(A, steps=40, seed=0, precision="f64"):
    """(min, max) Ritz values of a `steps`-step Lanczos run on the row-distributed
    operator (dot products all-reduced; the start vector's rows are drawn per
    rank)."""
    comm = A.comm
    prec = 32 if precision == "mixed" else 64
    dt = torch.float64 if prec == 64 else torch.float32
    dev = A.device
    g = torch.Generator(device=dev)
    g.manual_seed(seed * 1000003 + comm.rank)
    v = torch.rand((A.n_local, 1), generator=g, dtype=torch.float64, device=dev) - 0.5
    v /= _colnorms(comm, v)
    al, be = [], []
    v0 = torch.zeros_like(v)
    b_prev = 0.0
    for i in range(steps + 1):
        f = A.matmul(v.to(dt), prec=prec).to(torch.float64)
        if i:
            f -= b_prev * v0
        a = float(_gram(comm, v, f).item())
        f -= a * v
        al.append(a)
        if i == steps:
            break
        b = float(_colnorms(comm, f).item())
        if b == 0.0:
            break
        be.append(b)
        v0, v = v, f / b
        b_prev = b
    T = np.diag(al) + np.diag(be[:len(al) - 1], -1) + np.diag(be[:len(al) - 1], 1)
    w = np.linalg.eigvalsh(T)
    return float(w.min()), float(w.max())


def chfsi_rowblock(A: RowBlockOperator, k, tol=1e-6, Q=None, precision="mixed", degree=24, guard=None,
                   maxiter=300, seed=0, final_f64=True, return_info=False):
    """Lowest k eigenpairs of H (+PlusI) orthogonal to the rows of Q, on the
    row-distributed operator A; the iteration of solvers.chfsi.chfsi (scaled
    Chebyshev filter, projections, Cholesky-QR twice, Rayleigh-Ritz, locking at
    ||H y - theta y|| <= tol ||H||, the locked + active restart after
    STALL_RESTART iterations without a lock, a final FP64 Rayleigh-Ritz).

    Q: this rank's columns (r, 3 (b - a)) of a globally orthonormal row basis.
    Returns (eigenvalues (k,) ascending, this rank's rows (3 (b - a), k) of the
    eigenvectors), FP64 on A's device; every rank gets the same eigenvalues."""
    t_start = time.perf_counter()
    comm = A.comm
    n, n_loc, dev = A.shape[0], A.n_local, A.device
    if not 0 < k < n:
        raise AssertionError("ABORTED. k must be in (0, n)")
    if precision not in ("f64", "mixed"):
        raise AssertionError("ABORTED. precision must be 'f64' or 'mixed'")
    prec = 32 if precision == "mixed" else 64
    guard = default_guard(k) if guard is None else guard
    p = min(k + guard, n - (0 if Q is None else Q.shape[0]))
    Qd = None if Q is None else Q.to(device=dev, dtype=torch.float64).contiguous()
    lo, hi = spectrum_bound(A, steps=40, seed=seed + 1, precision=precision)
    b_up = hi * 1.02 + 1e-3 * abs(hi)
    normH = b_up
    g = torch.Generator(device=dev)
    g.manual_seed(seed * 1000003 + 7 + comm.rank)
    Y = torch.randn((n_loc, p), generator=g, dtype=torch.float64, device=dev)
    Y = _cholqr(comm, _project_out(comm, Y, Qd), n)
    th, Y, HY = _rr(comm, A, Y, prec)
    filt = _RowFilter(A, prec)
    locked = torch.empty((0, n_loc), dtype=torch.float64, device=dev)
    locked_theta = []
    it, n_rr, n_restarts, stall = 0, 1, 0, 0
    for it in range(maxiter):
        R = HY - Y * torch.from_numpy(th).to(dev)[None, :]
        res = _colnorms(comm, R).cpu().numpy()
        want = k - locked.shape[0]
        nl = 0
        while nl < min(want, Y.shape[1]) and res[nl] <= tol * normH:
            nl += 1
        if nl:
            locked = torch.cat([locked, Y[:, :nl].t()], dim=0)
            locked_theta.extend(th[:nl].tolist())
            Y, HY, th = Y[:, nl:], HY[:, nl:], th[nl:]
        if locked.shape[0] >= k:
            break
        stall = 0 if nl else stall + 1
        if stall >= STALL_RESTART and locked.shape[0]:
            th, Y, HY = _rr(comm, A, torch.cat([locked.t(), Y], dim=1), prec)
            locked = locked[:0]
            locked_theta = []
            n_rr += 1
            n_restarts += 1
            stall = 0
            continue
        a = float(th[-1])
        a0 = float(min(th[0], locked_theta[0] if locked_theta else th[0]))
        if not (a0 < a < b_up):
            a0 = a - 1e-3 * abs(a)
        Z = filt(Y, degree, a, b_up, a0 - 1e-12)
        Z = _project_out(comm, Z, Qd)
        Z = _project_out(comm, Z, locked)
        Z = _cholqr(comm, Z, n)
        th, Y, HY = _rr(comm, A, Z, prec)
        n_rr += 1
    converged = locked.shape[0] >= k
    if not converged:
        extra = k - locked.shape[0]
        locked = torch.cat([locked, Y[:, :extra].t()], dim=0)
        locked_theta.extend(th[:extra].tolist())
    L = locked[:k].t().contiguous()
    final_res = None
    if final_f64:
        th_f, L, HL = _rr(comm, A, L, 64)
        final_res = (_colnorms(comm, HL - L * torch.from_numpy(th_f).to(dev)[None, :]).cpu().numpy() / normH)
        evals = th_f
    else:
        evals = np.asarray(locked_theta[:k])
        idx = np.argsort(evals)
        evals = evals[idx]
        L = L[:, torch.from_numpy(idx).to(dev)]
    evals_t = torch.from_numpy(np.ascontiguousarray(evals)).to(dev)
    if return_info:
        info = dict(iterations=it + 1, converged=converged, n_spmm=A.n_spmm, n_spmm_filter=filt.n_spmm, n_rr=n_rr,
                    lock_restarts=n_restarts, normH=normH, degree=degree, block=p, halo_bytes=A.halo_bytes,
                    max_rel_residual=None if final_res is None else float(final_res.max()),
                    seconds=time.perf_counter() - t_start)
        return evals_t, L, info
    return evals_t, L


def gather_rows(comm, V_local, parts, dst=0):
    """The full (3N, k) array on rank dst (None elsewhere), from every rank's rows."""
    if comm.world == 1:
        return V_local
    if comm.rank == dst:
        full = torch.empty((3 * parts[-1][1],) + tuple(V_local.shape[1:]), dtype=V_local.dtype,
                           device=V_local.device)
        a, b = parts[dst]
        full[3 * a:3 * b] = V_local
        comm.p2p([], [(r, full[3 * parts[r][0]:3 * parts[r][1]]) for r in range(comm.world) if r != dst])
        return full
    comm.p2p([(dst, V_local.contiguous())], [])
    return None


def rowblock_normal_modes(X_nm: torch.Tensor, k: int, *, rc_gamma_A=8.0, plus_i=1.0, precision="mixed", tol=1e-6,
                          seed=0, group=None, gather=True, **kw):
    """Lowest k non-rigid modes of one structure with its Hessian rows split over
    the ranks of `group` (one GPU each, made current with torch.cuda.set_device
    before the process group's first call, as NCCL point-to-point needs; X_nm the
    same (N, 3) float64 nm coordinates on every rank, on that rank's GPU).

    Every rank orders the atoms (Cuthill-McKee) and builds the neighbour lists of
    the whole structure itself (the same inputs give the same lists), keeps the
    store rows of its own range, and runs chfsi_rowblock.  Returns (eigval (k,)
    with PlusI removed, eigvec (k, N, 3) in input atom order on rank 0 -- None on
    the others, or this rank's rows with gather=False --, info)."""
    from . import _native, graph
    from .deflation import rigid_body_basis
    comm = RowBlockComm(group)
    t0 = time.perf_counter()
    order, undo = graph.cuthill_mckee(X_nm, rc_gamma_A)
    Xr = X_nm[order].contiguous()
    degree, rowptr, cols = _native.neighbor_lists(Xr, rc_gamma_A / 10.0)
    parts = row_partition(rowptr, comm.world)
    ranges = halo_ranges(rowptr, cols, parts)
    a, b = parts[comm.rank]
    lo, hi = ranges[comm.rank]
    precisions = ("f64", "f32") if precision == "mixed" else ("f64",)
    local = StoreRows(Xr, rc_gamma_A, plus_i, rowptr, cols, a, b, lo, hi, precisions)
    del degree, rowptr, cols
    A = RowBlockOperator(local, parts, ranges, comm, Xr.shape[0], Xr.device)
    Q = rigid_body_basis(Xr)[:, 3 * a:3 * b]
    setup = time.perf_counter() - t0
    ev, V, info = chfsi_rowblock(A, k, tol=tol, Q=Q, precision=precision, seed=seed, return_info=True, **kw)
    info.update(dict(parts=parts, ranges=ranges, setup_s=setup, local_nnz_blocks=local.nnz_blocks))
    if not gather:
        return ev - plus_i, V, info
    full = gather_rows(comm, V, parts)
    if full is None:
        return ev - plus_i, None, info
    modes = full.t().reshape(k, Xr.shape[0], 3)[:, undo, :]
    return ev - plus_i, modes, info
