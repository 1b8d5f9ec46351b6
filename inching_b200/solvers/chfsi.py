"""Block Chebyshev-filtered subspace iteration with locking and explicit deflation
(the many-mode solver of this package; no single reference function).

It computes the same quantity as the reference's filtered TRLM ("CTRLM",
InchingLiteInteger/Burn/ThickRestartLanczosHotellingDeflation/T1.py with
User_PolynomialParams, driven window by window in
Notebook/Application/04_Inching_EigenproblemManyCTRLM.ipynb): the lowest k
non-rigid modes of H + PlusI*I.  Instead of one vector at a time it filters a
whole block, so every Hessian application is a multivector SpMM and every
projection a tall-skinny GEMM:

  Y <- p_m(H) Y        scaled Chebyshev filter damping [a, b] (a = largest Ritz
                       value of the block, b = spectrum upper bound), one fused
                       SpMM per degree (Zhou & Saad, J. Comput. Phys. 219 (2006),
                       Alg. "Chebyshev filter with scaling")
  Y <- Y - Q Q^T Y     explicit deflation of the rigid-body basis and of locked
                       modes (FP64 GEMMs)
  Y <- orth(Y)         Cholesky-QR twice (FP64)
  Rayleigh-Ritz        G = Y^T H Y, eigh (FP64), rotate; residuals ||H y - theta y||
  lock                 leading Ritz pairs with residual <= tol * ||H||; after
                       STALL_RESTART iterations without a new lock, one
                       Rayleigh-Ritz over locked + active vectors and locking
                       starts again (see the loop)

precision="mixed": filter and in-loop Rayleigh-Ritz products on the FP32 store
with FP32 blocks; projections, orthonormalisation, the small eigenproblems and
a final FP64 Rayleigh-Ritz + residual pass over the locked modes in FP64.
precision="f64": everything FP64.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from ..krylov import HessianOperator
from ..spectrum import estimate_spectrum_bound


STALL_RESTART = 3    # iterations without a new lock before the locked + active Rayleigh-Ritz


def autotune_store(A, precs):
    """Time the wide-product launch choices once for this store (cached per store
    size) at each precision the solver uses; no-op for operators that are not
    Hessian stores on the GPU."""
    if getattr(A, "spmm_cfg", None) is None or getattr(A, "device", None) is None or A.device.type != "cuda":
        return
    from ..autotune import tune_spmm
    for prec in precs:
        if A.has(prec):
            tune_spmm(A, 128 if prec == 32 else 64, prec=prec)


def default_guard(k):
    """Guard vectors carried beyond the k wanted ones (a quarter of k, at least 16:
    the gap to the block's last Ritz value sets the filter's convergence rate)."""
    return max(16, int(math.ceil(0.25 * k)))


def _cholqr(Y):
    """Orthonormalise columns of Y (FP64) by Cholesky-QR applied twice.  The
    triangular factor is inverted on the small (p, p) side so that the tall
    update is one GEMM; Householder QR if the Gram matrix is not positive."""
    for _ in range(2):
        G = Y.t() @ Y
        R, info = torch.linalg.cholesky_ex(G, upper=True)
        if int(info) != 0:
            Qf, _ = torch.linalg.qr(Y)
            return Qf
        Rinv = torch.linalg.solve_triangular(R, torch.eye(R.shape[0], dtype=R.dtype, device=R.device), upper=True)
        Y = Y @ Rinv
    return Y


def _project_out(Y, B):
    """Y <- Y - B^T (B Y) for row-basis B (r, n), twice."""
    if B is None or B.shape[0] == 0:
        return Y
    for _ in range(2):
        Y = Y - B.t() @ (B @ Y)
    return Y


class _Filter:
    def __init__(self, A, prec):
        self.A = A
        self.prec = prec
        self.n_spmm = 0

    def __call__(self, X64, m, a, b, a0, degrees=None):
        """Scaled Chebyshev filter of degree m on [a, b] normalised at a0 < a; with
        `degrees` (one per column, each in [1, m]) column i stops after degrees[i]."""
        if degrees is not None:
            return self._per_column(X64, m, a, b, a0, degrees)
        dt = torch.float64 if self.prec == 64 else torch.float32
        e = (b - a) / 2.0
        c = (b + a) / 2.0
        sigma = e / (a0 - c)
        sigma1 = sigma
        tau = 2.0 / sigma1
        b = X64.shape[1]
        bp = (b + 7) // 8 * 8          # aligned width for the vector-gather SpMM
        X = torch.zeros((X64.shape[0], bp), dtype=dt, device=X64.device)
        X[:, :b] = X64                 # fresh buffer: the recurrence overwrites X
        Y = torch.empty_like(X)
        self.A.matmul(X, out=Y, prec=self.prec, alpha=sigma1 / e, gamma=-sigma1 * c / e)
        self.n_spmm += 1
        for _ in range(2, m + 1):
            s2 = 1.0 / (tau - sigma)
            # X <- 2 s2/e (H Y - c Y) - sigma s2 X, written over X, then swap
            self.A.matmul(Y, out=X, prec=self.prec, alpha=2.0 * s2 / e, gamma=-2.0 * s2 * c / e,
                          beta=-sigma * s2, Yin=X)
            X, Y = Y, X
            sigma = s2
            self.n_spmm += 1
        return Y[:, :b].to(torch.float64)

    def _per_column(self, X64, m, a, b, a0, degrees):
        """The same recurrence with per-column degrees: columns sorted by degree, the
        SpMM runs on the suffix of columns still going (start rounded down to a
        multiple of 8, so rows stay aligned), and each column's value is taken at
        its own last step."""
        dt = torch.float64 if self.prec == 64 else torch.float32
        nb = X64.shape[1]
        deg = np.clip(np.asarray(degrees, dtype=np.int64), 1, m)
        order = np.argsort(deg, kind="stable")
        deg_s = deg[order]
        order_t = torch.from_numpy(order).to(X64.device)
        e = (b - a) / 2.0
        c = (b + a) / 2.0
        sigma = e / (a0 - c)
        sigma1 = sigma
        tau = 2.0 / sigma1
        bp = (nb + 7) // 8 * 8
        X = torch.zeros((X64.shape[0], bp), dtype=dt, device=X64.device)
        X[:, :nb] = X64.index_select(1, order_t)
        Y = torch.empty_like(X)
        out = torch.empty((X64.shape[0], nb), dtype=torch.float64, device=X64.device)
        self.A.matmul(X, out=Y, prec=self.prec, alpha=sigma1 / e, gamma=-sigma1 * c / e)
        self.n_spmm += 1
        self.col_steps = getattr(self, "col_steps", 0) + bp
        done = 0
        for t in range(1, int(deg_s[-1]) + 1):
            if t > 1:
                s0 = (done // 8) * 8
                s2 = 1.0 / (tau - sigma)
                self.A.matmul(Y[:, s0:], out=X[:, s0:], prec=self.prec, alpha=2.0 * s2 / e,
                              gamma=-2.0 * s2 * c / e, beta=-sigma * s2, Yin=X[:, s0:])
                X, Y = Y, X
                sigma = s2
                self.n_spmm += 1
                self.col_steps += bp - s0
            end = int(np.searchsorted(deg_s, t, side="right"))
            if end > done:
                out[:, done:end] = Y[:, done:end]
                done = end
        res = torch.empty_like(out)
        res[:, order_t] = out
        return res


def chebyshev_degrees(theta, res, n_wanted, tol_abs, a, b, m, margin=2, floor=2):
    """Per-vector filter degrees (Berljafa, Wortmann & Di Napoli, ChASE, 2015): a
    wanted vector with Ritz value theta and residual r needs about
    log(r / tol) / log(1 / rho) further steps, rho = |t| - sqrt(t^2 - 1) the
    per-step damping of [a, b] relative to theta, t = (theta - c) / e.  Wanted
    vectors get that (+ margin, within [floor, m]); guard vectors keep m."""
    theta = np.asarray(theta, dtype=np.float64)
    e = (b - a) / 2.0
    c = (b + a) / 2.0
    t = np.abs((theta - c) / e)
    rho = np.where(t > 1.0, t - np.sqrt(np.maximum(t * t - 1.0, 0.0)), 1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        need = np.log(np.maximum(np.asarray(res) / tol_abs, 1.0)) / np.maximum(-np.log(rho), 1e-12)
    deg = np.full(len(theta), m, dtype=np.int64)
    w = min(n_wanted, len(theta))
    deg[:w] = np.clip(np.ceil(need[:w]).astype(np.int64) + margin, floor, m)
    return deg


class _GraphFilter:
    """The scaled Chebyshev filter of _Filter, captured as one CUDA graph per block
    width: its m SpMM launches read their coefficients from a device table (the
    segmented epilogue with a single segment), so a new filter interval only
    rewrites that table and the whole filter replays as one graph launch."""

    def __init__(self, A, prec):
        self.A = A
        self.prec = prec
        self.n_spmm = 0
        self.graphs = {}
        self.seg = torch.zeros(A.n_atoms, dtype=torch.int32, device=A.device)
        self.replays = 0

    def _build(self, bp, m):
        dt = torch.float64 if self.prec == 64 else torch.float32
        n = self.A.shape[0]
        X = torch.zeros((n, bp), dtype=dt, device=self.A.device)
        Y = torch.zeros_like(X)
        table = torch.zeros((m, 1, 3), dtype=torch.float64, device=self.A.device)
        out = {"X": X, "Y": Y, "table": table}

        def body():
            x, y = X, Y
            self.A.matmul_seg(x, y, self.seg, table[0], prec=self.prec)
            for t in range(1, m):
                self.A.matmul_seg(y, x, self.seg, table[t], Yin=x, prec=self.prec)
                x, y = y, x
            out["res"] = y

        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            body()                                  # warm-up outside capture
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            body()
        out["graph"] = g
        return out

    def __call__(self, X64, m, a, b, a0):
        e = (b - a) / 2.0
        c = (b + a) / 2.0
        sigma = e / (a0 - c)
        sigma1 = sigma
        tau = 2.0 / sigma1
        rows = [[sigma1 / e, -sigma1 * c / e, 0.0]]
        for _ in range(2, m + 1):
            s2 = 1.0 / (tau - sigma)
            rows.append([2.0 * s2 / e, -2.0 * s2 * c / e, -sigma * s2])
            sigma = s2
        return self.run_rows(X64, rows)

    def run_rows(self, X64, rows):
        """Any three-term recurrence X_1 = a_0 H X_0 + g_0 X_0,
        X_{t+1} = a_t H X_t + g_t X_t + b_t X_{t-1}; rows[t] = (a_t, g_t, b_t)."""
        m = len(rows)
        nb = X64.shape[1]
        bp = (nb + 7) // 8 * 8
        key = (bp, m)
        if key not in self.graphs:
            self.graphs[key] = self._build(bp, m)
        gph = self.graphs[key]
        gph["table"].copy_(torch.tensor(rows, dtype=torch.float64).reshape(m, 1, 3))
        gph["X"].zero_()
        gph["X"][:, :nb] = X64
        gph["graph"].replay()
        self.n_spmm += m
        self.replays += 1
        return gph["res"][:, :nb].to(torch.float64)


DEVICE_EIGH_MIN = 64   # projected matrices at least this large are diagonalised on the GPU


def eigh_sym(G):
    """Eigenpairs of the symmetric FP64 device matrix G: (theta ascending as numpy,
    eigenvectors as a device tensor).  From DEVICE_EIGH_MIN rows on, cuSOLVER on the
    device (320 x 320: 3.4 ms against 9 ms for host LAPACK on this machine, no
    round trip of G and W); smaller ones on the host."""
    if G.shape[0] >= DEVICE_EIGH_MIN:
        th, W = torch.linalg.eigh(G)
        return th.cpu().numpy(), W
    th, W = np.linalg.eigh(G.cpu().numpy())
    return th, torch.from_numpy(W).to(G.device)


def _rr(A, Y, prec):
    """Rayleigh-Ritz on orthonormal Y (n, p): returns theta (asc, numpy), Y W, (H Y) W."""
    if prec == 64:
        HY = A.matmul(Y.contiguous(), prec=64)
    else:
        HY = A.matmul(Y.to(torch.float32).contiguous(), prec=32).to(torch.float64)
    G = Y.t() @ HY
    G = 0.5 * (G + G.t())
    th, Wd = eigh_sym(G)
    return th, Y @ Wd, HY @ Wd


class _Phases:
    """CUDA-event timing of the solver phases (enabled with profile=True)."""

    def __init__(self, on):
        self.on = on
        self.ev = {}

    def __call__(self, name):
        return _Span(self, name)

    def summary(self):
        if not self.on:
            return None
        torch.cuda.synchronize()
        return {k: round(sum(a.elapsed_time(b) for a, b in v), 2) for k, v in self.ev.items()}


class _Span:
    def __init__(self, ph, name):
        self.ph, self.name = ph, name

    def __enter__(self):
        if self.ph.on:
            self.a = torch.cuda.Event(enable_timing=True)
            self.a.record()

    def __exit__(self, *x):
        if self.ph.on:
            b = torch.cuda.Event(enable_timing=True)
            b.record()
            self.ph.ev.setdefault(self.name, []).append((self.a, b))


def chfsi(A, k, tol=1e-6, Q=None, precision="mixed", degree=24, guard=None, maxiter=300, X0=None, seed=0,
          spectrum_upper=None, final_f64=True, verbose=False, return_info=False, profile=False, cuda_graph=False,
          adaptive_degree=False, return_block=False):
    """Lowest k eigenpairs of A (+PlusI) orthogonal to the rows of Q.

    tol is relative: a pair is locked when ||H y - theta y|| <= tol * ||H||, with
    ||H|| estimated by the Lanczos upper bound of the spectrum.
    Returns (eigenvalues (k,) ascending, eigenvectors (n, k)) as FP64 CUDA tensors.
    With return_block, the eigenvector array is the whole (n, k + guard) block:
    the k locked modes followed by the unconverged Ritz vectors of the last
    Rayleigh-Ritz step, all orthonormal (an initial block for a finer solve)."""
    t_start = time.perf_counter()
    n = A.shape[0]
    dev = A.device
    assert 0 < k < n, "ABORTED. k must be in (0, n)"
    assert precision in ("f64", "mixed"), "ABORTED. precision must be 'f64' or 'mixed'"
    prec = 32 if precision == "mixed" else 64
    if guard is None:
        guard = default_guard(k)
    p = min(k + guard, n - (0 if Q is None else Q.shape[0]))
    Qd = None if Q is None else HessianOperator(A, Q=Q).Q
    ph = _Phases(profile)
    with ph("autotune"):
        autotune_store(A, sorted({prec, 64}))
    if spectrum_upper is None:
        with ph("bound"):
            lo, hi = estimate_spectrum_bound(A, steps=40, seed=seed + 1, precision=precision)
        spectrum_upper = hi * 1.02 + 1e-3 * abs(hi)
    b_up = float(spectrum_upper)
    normH = b_up
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    Y = torch.randn((n, p), generator=g, dtype=torch.float64, device=dev)
    if X0 is not None:
        X0 = X0.to(device=dev, dtype=torch.float64)
        c0 = min(X0.shape[1], p)
        Y[:, :c0] = X0[:, :c0]
    with ph("orth"):
        Y = _cholqr(_project_out(Y, Qd))
    with ph("rr"):
        th, Y, HY = _rr(A, Y, prec)
    filt = _GraphFilter(A, prec) if (cuda_graph and hasattr(A, "matmul_seg")) else _Filter(A, prec)
    locked = torch.empty((0, n), dtype=torch.float64, device=dev)   # rows
    locked_theta = []
    it = 0
    n_rr = 1
    n_restarts = 0
    stall = 0
    res = np.full(p, np.inf)
    for it in range(maxiter):
        with ph("residual"):
            R = HY - Y * torch.from_numpy(th).to(dev)[None, :]
            res = torch.linalg.vector_norm(R, dim=0).cpu().numpy()
        want = k - locked.shape[0]
        nl = 0
        while nl < min(want, Y.shape[1]) and res[nl] <= tol * normH:
            nl += 1
        if nl:
            locked = torch.cat([locked, Y[:, :nl].t()], dim=0)
            locked_theta.extend(th[:nl].tolist())
            Y, HY, th = Y[:, nl:], HY[:, nl:], th[nl:]
        if verbose:
            print(f"it {it} locked {locked.shape[0]}/{k} maxres(active wanted) "
                  f"{res[nl:want].max() / normH if want > nl else 0:.2e} a={th[-1]:.4f}")
        if locked.shape[0] >= k:
            break
        stall = 0 if nl else stall + 1
        if stall >= STALL_RESTART and locked.shape[0]:
            # A locked vector is only accurate to tol; inside a cluster whose gaps are
            # of the order of tol*||H|| it carries a sizeable share of unlocked
            # neighbours, and the active block (kept orthogonal to it) cannot get
            # below tol.  One Rayleigh-Ritz over locked + active resolves that
            # coupling; locking then starts again from the new Ritz pairs.
            with ph("rr"):
                th, Y, HY = _rr(A, torch.cat([locked.t(), Y], dim=1), prec)
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
        with ph("filter"):
            if adaptive_degree and it > 0 and not isinstance(filt, _GraphFilter):
                degs = chebyshev_degrees(th, res[nl:nl + len(th)], k - locked.shape[0], tol * normH, a, b_up,
                                         degree)
                Z = filt(Y, degree, a, b_up, a0 - 1e-12, degrees=degs)
            else:
                Z = filt(Y, degree, a, b_up, a0 - 1e-12)
        with ph("orth"):
            Z = _project_out(Z, Qd)
            Z = _project_out(Z, locked)
            Z = _cholqr(Z)
        with ph("rr"):
            th, Y, HY = _rr(A, Z, prec)
        n_rr += 1
    converged = locked.shape[0] >= k
    if not converged:
        print(f"ABORTED. chfsi did not converge in {maxiter} iterations: {locked.shape[0]} of {k} modes locked")
        extra = k - locked.shape[0]
        locked = torch.cat([locked, Y[:, :extra].t()], dim=0)
        locked_theta.extend(th[:extra].tolist())
    L = locked[:k].t().contiguous()
    if final_f64:
        with ph("final_f64"):
            th_f, L, HL = _rr(A, L, 64)
        R = HL - L * torch.from_numpy(th_f).to(dev)[None, :]
        final_res = torch.linalg.vector_norm(R, dim=0).cpu().numpy() / normH
        evals = th_f
    else:
        evals = np.asarray(locked_theta[:k])
        idx = np.argsort(evals)
        evals = evals[idx]
        L = L[:, torch.from_numpy(idx).to(dev)]
        final_res = None
    if return_block:
        # the active block holds p - (modes locked before the exit) columns; after a
        # non-converged exit its leading ones were appended to the locked set, so the
        # unused Ritz vectors are always its trailing p - k columns
        L = torch.cat([L, Y[:, Y.shape[1] - (p - k):]], dim=1)
    evals_t = torch.from_numpy(np.ascontiguousarray(evals)).to(dev)
    if return_info:
        info = dict(iterations=it + 1, converged=converged, n_spmm_filter=filt.n_spmm, n_rr=n_rr,
                    filter_graph_replays=getattr(filt, "replays", 0), lock_restarts=n_restarts,
                    filter_column_steps=getattr(filt, "col_steps", None),
                    normH=normH, degree=degree, block=p,
                    max_rel_residual=None if final_res is None else float(final_res.max()),
                    seconds=time.perf_counter() - t_start, phases_ms=ph.summary())
        return evals_t, L, info
    return evals_t, L


# ---------------------------------------------------------------------------
# Memory-lean variant for structures whose block does not fit several times in HBM
# ---------------------------------------------------------------------------
def _rows(n, rows):
    for r0 in range(0, n, rows):
        yield slice(r0, min(r0 + rows, n))


def lean_degree(A, p):
    """Filter degree of the memory-lean solver: each iteration costs tall GEMMs
    (~ n p^2, n dof) besides the filter's SpMMs (~ nnz p per degree, nnz stored
    blocks), so the wider the block relative to the matrix, the more filtering per
    iteration pays.  24 at p n / nnz <= 10 (256 modes of 100k atoms: 9.6), growing
    with the square root of that ratio, in multiples of 8 up to 64 (1,000 modes of
    2.4M atoms: ratio 37 -> 48, which took 4 iterations and 93 s against 10 and
    126 s at 24)."""
    nnz = getattr(A, "nnz_blocks", None)
    if not nnz:
        return 24
    ratio = p * A.shape[0] / nnz          # dof x block width / stored blocks
    d = 24.0 * math.sqrt(max(ratio, 10.0) / 10.0)
    return int(min(64, max(24, 8 * round(d / 8))))


def chfsi_lean(A, k, tol=1e-6, Q=None, precision="mixed", degree=None, guard=None, maxiter=100, X0=None, seed=0,
               chunk=256, row_chunk=1 << 20, window=512, verbose=False, return_info=False, profile=False,
               fold_orth=True):
    """Same iteration as chfsi() with one (n, p) FP64 array B holding the locked
    modes (columns [0, L)) and the active block (columns [L, p)):

      * the filter runs on column chunks of `chunk` vectors (it acts column by
        column), with FP32 (or FP64) buffers of that width only;
      * Rayleigh-Ritz forms G = Y^T H Y chunk by chunk (H Y on the FP32 store in
        mixed precision, FP64 otherwise), so H Y is never stored; explicit FP64
        residuals are taken for the leading `window` wanted active columns, the
        only ones that can lock next;
      * rotations, projections and Cholesky-QR update B in row chunks; with
        fold_orth (default) the second Cholesky-QR pass's factor is folded into
        the Rayleigh-Ritz rotation (see orth());
      * converged leading active columns become locked by moving L.
    Peak memory is about n*p*8 bytes plus a few (n, chunk) buffers: the 2.4M-atom,
    1000-mode configuration (n = 7.2M, p = 1250) needs ~72 GB for B.  A contiguous
    FP64 X0 of shape (n, p) is used in place as B (it is overwritten)."""
    t_start = time.perf_counter()
    n = A.shape[0]
    dev = A.device
    prec = 32 if precision == "mixed" else 64
    if guard is None:
        guard = default_guard(k)
    p = min(k + guard, n - (0 if Q is None else Q.shape[0]))
    if degree is None:
        degree = lean_degree(A, p)
    Qd = None if Q is None else HessianOperator(A, Q=Q).Q
    autotune_store(A, sorted({prec, 64}))
    lo, hi = estimate_spectrum_bound(A, steps=40, seed=seed + 1, precision=precision)
    b_up = hi * 1.02 + 1e-3 * abs(hi)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    if (X0 is not None and X0.dtype == torch.float64 and X0.is_contiguous() and tuple(X0.shape) == (n, p)
            and X0.device == dev):
        B = X0          # take over the caller's block: no second n x p copy
    else:
        B = torch.empty((n, p), dtype=torch.float64, device=dev)
        c0 = 0 if X0 is None else min(X0.shape[1], p)
        for cs in range(0, p, chunk):
            ce = min(cs + chunk, p)
            if ce <= c0:
                B[:, cs:ce] = X0[:, cs:ce].to(torch.float64)
            else:
                B[:, cs:ce] = torch.randn((n, ce - cs), generator=g, dtype=torch.float64, device=dev)
                if cs < c0:
                    B[:, cs:c0] = X0[:, cs:c0].to(torch.float64)

    def project(L):
        """Active columns minus their components along Q (rigid) and B[:, :L]."""
        act = slice(L, p)
        for _ in range(2):
            for basis in ((Qd.t() if Qd is not None else None), (B[:, :L] if L > 0 else None)):
                if basis is None:
                    continue
                C = basis.t() @ B[:, act]                         # (r, A) small
                for rs in _rows(n, row_chunk):
                    B[rs, act] -= basis[rs] @ C

    def orth_f64_pass(act):
        G = B[:, act].t() @ B[:, act]
        R, info = torch.linalg.cholesky_ex(G, upper=True)
        if int(info) != 0:
            raise RuntimeError("chfsi_lean: Gram matrix not positive definite")
        Rinv = torch.linalg.solve_triangular(R, torch.eye(R.shape[0], dtype=R.dtype, device=dev), upper=True)
        for rs in _rows(n, row_chunk):
            B[rs, act] = B[rs, act] @ Rinv

    def orth(L):
        """Cholesky-QR of the active block.  With fold_orth, one FP64 pass (Gram,
        Cholesky, rotation) and then the second pass's FP64 Gram only: its factor
        R2 is returned instead of applied, and the Rayleigh-Ritz step folds R2^-1
        into its rotation (one tall rotation fewer per iteration).  Returns R2, or
        None when the block is left orthonormal (two full passes)."""
        act = slice(L, p)
        orth_f64_pass(act)
        if not fold_orth:
            orth_f64_pass(act)
            return None
        G2 = B[:, act].t() @ B[:, act]
        R2, info = torch.linalg.cholesky_ex(G2, upper=True)
        if int(info) != 0:
            raise RuntimeError("chfsi_lean: Gram matrix not positive definite")
        return R2

    def rayleigh_ritz(L, R2=None):
        """Rotate the active block to Ritz vectors; returns (theta, residual norms).
        Explicit FP64 residuals are computed for the leading `window` wanted active
        columns only (locking proceeds from the front); the others report inf.
        With R2 (upper triangular) the active block Y is not orthonormal but Y R2^-1
        is: the projected matrix becomes R2^-T (Y^T H Y) R2^-1 and the rotation
        R2^-1 W."""
        act_n = p - L
        G = torch.zeros((act_n, act_n), dtype=torch.float64, device=dev)
        for cs in range(L, p, chunk):
            ce = min(cs + chunk, p)
            with ph("rr_spmm"):
                if prec == 32:
                    # in-loop Rayleigh-Ritz on the FP32 store, as chfsi() does: the FP64
                    # residuals below decide locking and the final pass is FP64 throughout
                    HYc = A.matmul(B[:, cs:ce].to(torch.float32).contiguous(), prec=32).to(torch.float64)
                else:
                    HYc = A.matmul(B[:, cs:ce].contiguous(), prec=64)
            with ph("rr_gram"):
                G[:, cs - L:ce - L] = B[:, L:].t() @ HYc
            del HYc
        G = 0.5 * (G + G.t())
        if R2 is not None:
            Rinv = torch.linalg.solve_triangular(R2, torch.eye(R2.shape[0], dtype=R2.dtype, device=dev), upper=True)
            G = Rinv.t() @ G @ Rinv
            G = 0.5 * (G + G.t())
        with ph("rr_eigh"):
            th, Wd = eigh_sym(G)
        if R2 is not None:
            Wd = Rinv @ Wd
        with ph("rr_rotate"):
            for rs in _rows(n, row_chunk):
                B[rs, L:] = B[rs, L:] @ Wd
        res = np.full(len(th), np.inf)
        last = min(len(th), k - L, window)
        thd = torch.from_numpy(th[:last].copy()).to(dev)
        with ph("rr_residual"):
            for cs in range(0, last, chunk):
                ce = min(cs + chunk, last)
                Yc = B[:, L + cs:L + ce].contiguous()
                R = A.matmul(Yc, prec=64) - Yc * thd[cs:ce][None, :]
                res[cs:ce] = torch.linalg.vector_norm(R, dim=0).cpu().numpy()
        return th, res

    ph = _Phases(profile)
    with ph("project"):
        project(0)
    with ph("orth"):
        R2 = orth(0)
    with ph("rr"):
        th, res = rayleigh_ritz(0, R2)
    L = 0
    locked_theta = []
    filt = _Filter(A, prec)
    it = 0
    stall = 0
    n_restarts = 0
    for it in range(maxiter):
        nl = 0
        while L + nl < k and nl < len(th) and res[nl] <= tol * b_up:
            nl += 1
        if nl:
            locked_theta.extend(th[:nl].tolist())
            th, res = th[nl:], res[nl:]
            L += nl
        if verbose:
            print(f"lean it {it}: locked {L}/{k}, max active res {res[:max(k - L, 1)].max() / b_up:.2e}")
        if L >= k:
            break
        stall = 0 if nl else stall + 1
        if stall >= STALL_RESTART and L:
            # locked + active Rayleigh-Ritz, as in chfsi(): clears the coupling of
            # the active block to modes locked inside a tight cluster
            with ph("rr"):
                th, res = rayleigh_ritz(0)
            L = 0
            locked_theta = []
            stall = 0
            n_restarts += 1
            continue
        a = float(th[-1])
        a0 = float(th[0])
        if not (a0 < a < b_up):
            a0 = a - 1e-3 * abs(a)
        with ph("filter"):
            for cs in range(L, p, chunk):
                ce = min(cs + chunk, p)
                B[:, cs:ce] = filt(B[:, cs:ce], degree, a, b_up, a0 - 1e-12)
        with ph("project"):
            project(L)
        with ph("orth"):
            R2 = orth(L)
        with ph("rr"):
            th, res = rayleigh_ritz(L, R2)
    converged = L >= k
    # final FP64 Rayleigh-Ritz over the first k columns, explicit residuals
    ph_final = ph("final_f64")
    ph_final.__enter__()
    Lk = B[:, :k]
    G = torch.zeros((k, k), dtype=torch.float64, device=dev)
    for cs in range(0, k, chunk):
        ce = min(cs + chunk, k)
        G[:, cs:ce] = Lk.t() @ A.matmul(Lk[:, cs:ce].contiguous(), prec=64)
    G = 0.5 * (G + G.t())
    thf, Wd = eigh_sym(G)
    for rs in _rows(n, row_chunk):
        B[rs, :k] = B[rs, :k] @ Wd
    thd = torch.from_numpy(thf).to(dev)
    worst = 0.0
    for cs in range(0, k, chunk):
        ce = min(cs + chunk, k)
        R = A.matmul(B[:, cs:ce].contiguous(), prec=64) - B[:, cs:ce] * thd[cs:ce][None, :]
        worst = max(worst, float(torch.linalg.vector_norm(R, dim=0).max()) / b_up)
    ph_final.__exit__(None, None, None)
    evals = torch.from_numpy(thf.copy()).to(dev)
    V = B[:, :k]
    if return_info:
        return evals, V, dict(iterations=it + 1, converged=converged, n_spmm_filter=filt.n_spmm, block=p,
                              degree=degree, normH=b_up, max_rel_residual=worst, lock_restarts=n_restarts,
                              seconds=time.perf_counter() - t_start, phases_ms=ph.summary())
    return evals, V
