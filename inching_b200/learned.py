"""Learned warm start: a message-passing network on the coarse bead graph that
sets the bead model's spring constants (no reference counterpart).

The bead model of inching_b200.warmstart (atoms pooled into ~6 A beads, bead
pairs within 12 A joined by springs) uses one spring constant for every pair.
Here a 3-layer message-passing network (width 128, FP32; messages averaged over
each bead's neighbours) reads the bead graph
-- node features: atoms per bead, bead radius of gyration, bead degree; edge
features: bead distance, number of atom-atom contacts across the pair -- and
predicts each pair's spring constant gamma_e = softplus(s_e) + 0.05.

Training (GPU): for a structure with lowest non-rigid eigenvalues lambda_t
computed by the plain FP64 solver, the loss is the mean squared log ratio
(log mu_t - log lambda_t)^2 of the bead model's lowest eigenvalues mu_t to them
(symmetric in over- and under-estimates; a squared relative error let the first
steps overshoot into the softplus floor).  d(loss)/d(gamma_e) is exact by
Hellmann-Feynman, d mu_t / d gamma_e = (u_e . (v_t[a] - v_t[b]))^2 with the
bead model's eigenvectors v_t, so no differentiation through the eigensolver is
needed.  The forward and backward passes are hand-written: graph gathers,
neighbour means, activations, the eigenvalue gradient and the Adam step are the
package's CUDA kernels (csrc/mpnn.cu); dense layers are cuBLAS GEMMs.

The prolonged block goes through a residual test against random columns (one
Rayleigh-Ritz each on the fine Hessian, over the leading 64 columns): if its
median Ritz residual is not lower, a random block is used.

Use: model = WarmStartMPNN.load(); X0 = learned_warm_start(X_nm, n_vectors, model),
or normal_modes(..., warm_start="learned") with the shipped weights.
"""
from __future__ import annotations

import math
import os

import numpy as np
import torch

from . import _native
from .deflation import rigid_body_basis
from .hessian import HessianStore
from .warmstart import bead_model

WIDTH = 128
NODE_F = 4
EDGE_F = 4
LAYERS = 3
GAMMA_FLOOR = 0.05
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_mpnn.npz")


# ---------------------------------------------------------------------------
# Bead graph and features
# ---------------------------------------------------------------------------
class BeadGraph:
    """Beads of a structure, their adjacency (self included, for the Hessian) and
    the message-passing edges (self excluded, CSR by destination)."""

    def __init__(self, X_nm: torch.Tensor, fine_rowptr=None, fine_cols=None, bead_edge_A=6.0, rc_bead_A=12.0):
        dev = X_nm.device
        self.rc_nm = rc_bead_A / 10.0
        pos, bead = bead_model(X_nm, bead_edge_A)
        self.pos, self.bead = pos.contiguous(), bead
        nb = pos.shape[0]
        self.n = nb
        one = torch.ones(bead.shape[0], dtype=torch.float64, device=dev)
        cnt = torch.zeros(nb, dtype=torch.float64, device=dev).index_add_(0, bead, one)
        d2 = ((X_nm - pos[bead]) ** 2).sum(dim=1)
        rg = torch.sqrt(torch.zeros(nb, dtype=torch.float64, device=dev).index_add_(0, bead, d2) / cnt)
        self.degree, self.rowptr, self.cols = _native.neighbor_lists(self.pos, self.rc_nm)
        rows = torch.repeat_interleave(torch.arange(nb, device=dev), self.degree.long())
        self.self_mask = rows == self.cols.long()
        keep = ~self.self_mask
        self.dst = rows[keep].to(torch.int32).contiguous()
        self.src = self.cols[keep].contiguous()
        mp_deg = self.degree.long() - 1
        self.mp_rowptr = torch.zeros(nb + 1, dtype=torch.int64, device=dev)
        self.mp_rowptr[1:] = torch.cumsum(mp_deg, 0)
        self.E = int(self.src.shape[0])
        d = torch.linalg.vector_norm(pos[self.src.long()] - pos[self.dst.long()], dim=1)
        contacts = torch.zeros(self.E, dtype=torch.float64, device=dev)
        if fine_rowptr is not None:
            contacts = self._contacts(fine_rowptr, fine_cols, nb)
        self.x = torch.stack([cnt / 64.0, rg * 10.0, mp_deg.double() / 30.0, torch.ones_like(cnt)], dim=1).float()
        self.ef = torch.stack([d / self.rc_nm, contacts / 64.0, torch.clamp(self.rc_nm / d, max=10.0) / 10.0,
                               torch.ones_like(d)], dim=1).float().contiguous()
        self.x = self.x.contiguous()

    def _contacts(self, rowptr, cols, nb):
        """Atom-atom contacts (pairs within the atomic cutoff) between each bead pair."""
        dev = rowptr.device
        n_at = rowptr.shape[0] - 1
        arows = torch.repeat_interleave(torch.arange(n_at, device=dev), torch.diff(rowptr))
        ba = self.bead[arows]
        bb = self.bead[cols.long()]
        key = ba * nb + bb
        cross = ba != bb
        key = key[cross]
        uk, cnt = torch.unique(key, return_counts=True)
        ekey = self.dst.long() * nb + self.src.long()
        pos = torch.searchsorted(uk, ekey).clamp(max=uk.numel() - 1)
        hit = uk[pos] == ekey
        return torch.where(hit, cnt[pos].double(), torch.zeros_like(ekey, dtype=torch.float64))

    def adjacency_weights(self, gamma_mp: torch.Tensor) -> torch.Tensor:
        """Spring constant per adjacency entry (self entries get 1; their block is 0)."""
        w = torch.ones(self.cols.shape[0], dtype=torch.float64, device=gamma_mp.device)
        w[~self.self_mask] = gamma_mp
        return w.contiguous()


# ---------------------------------------------------------------------------
# The network
# ---------------------------------------------------------------------------
def _param_shapes():
    shapes = [("W0", (NODE_F, WIDTH)), ("b0", (WIDTH,))]
    for l in range(LAYERS):
        shapes += [(f"Wm{l}", (WIDTH + EDGE_F, WIDTH)), (f"bm{l}", (WIDTH,)),
                   (f"Wu{l}", (2 * WIDTH, WIDTH)), (f"bu{l}", (WIDTH,))]
    shapes += [("wo", (WIDTH + EDGE_F, 1)), ("bo", (1,))]
    return shapes


def _mm(A, B, out=None, accumulate=False):
    """A @ B (+ out) on the package's dense-layer kernel (FP32); A and B may be
    transposed views."""
    if out is None:
        out = torch.empty((A.shape[0], B.shape[1]), dtype=torch.float32, device=A.device)
    return _native.mp_gemm(A, B, out, 1.0 if accumulate else 0.0)


_ones = {}


def _colsum(Y, out):
    """out (1, F) += column sums of Y (rows, F), as ones^T Y on the same kernel."""
    r = Y.shape[0]
    o = _ones.get((Y.device, r))
    if o is None:
        o = torch.ones((1, r), dtype=torch.float32, device=Y.device)
        _ones[(Y.device, r)] = o
    return _native.mp_gemm(o, Y, out, 1.0)


class WarmStartMPNN:
    def __init__(self, device="cuda", seed=0):
        self.shapes = _param_shapes()
        n = sum(int(np.prod(s)) for _, s in self.shapes)
        self.flat = torch.zeros(n, dtype=torch.float32, device=device)
        self.grad = torch.zeros_like(self.flat)
        self.m1 = torch.zeros_like(self.flat)
        self.m2 = torch.zeros_like(self.flat)
        self.step = 0
        self.p, self.g = {}, {}
        off = 0
        for name, shp in self.shapes:
            k = int(np.prod(shp))
            self.p[name] = self.flat[off:off + k].view(shp)
            self.g[name] = self.grad[off:off + k].view(shp)
            off += k
        rng = np.random.default_rng(seed)
        for name, shp in self.shapes:
            if name.startswith("W") or name == "wo":
                fan_in = shp[0]
                scale = math.sqrt(2.0 / fan_in) * (0.01 if name == "wo" else 1.0)
                self.p[name].copy_(torch.from_numpy(rng.standard_normal(shp).astype(np.float32) * scale))
        # softplus(bo) + floor = 1: the untrained model is the uniform bead model
        self.p["bo"].fill_(float(np.log(np.expm1(1.0 - GAMMA_FLOOR))))

    # -- persistence -----------------------------------------------------------
    def state(self):
        return {name: self.p[name].detach().cpu().numpy() for name, _ in self.shapes}

    def save(self, path=WEIGHTS, **meta):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez_compressed(path, **self.state(), **{f"meta_{k}": np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path=WEIGHTS, device="cuda"):
        m = cls(device=device)
        d = np.load(path)
        for name, _ in m.shapes:
            m.p[name].copy_(torch.from_numpy(d[name]))
        return m

    # -- forward / backward ------------------------------------------------------
    def forward(self, G: BeadGraph):
        p = self.p
        c = {}
        h = _mm(G.x, p["W0"])
        _native.mp("bias_relu", h, p["b0"], G.n, WIDTH)
        c["h0"] = h
        hs = [h]
        for l in range(LAYERS):
            Z = torch.empty((G.E, WIDTH + EDGE_F), dtype=torch.float32, device=h.device)
            _native.mp("edge_concat", h, G.ef, G.src, G.E, WIDTH, EDGE_F, Z)
            A = _mm(Z, p[f"Wm{l}"])
            _native.mp("bias_relu", A, p[f"bm{l}"], G.E, WIDTH)
            M = torch.empty((G.n, WIDTH), dtype=torch.float32, device=h.device)
            _native.mp("segment_sum", A, G.mp_rowptr, G.n, WIDTH, M)
            U = torch.cat([h, M], dim=1)
            T = _mm(U, p[f"Wu{l}"])
            _native.mp("bias_relu", T, p[f"bu{l}"], G.n, WIDTH)
            c[l] = (Z, A, U, T)
            h = h + T
            hs.append(h)
        R = torch.empty((G.E, WIDTH + EDGE_F), dtype=torch.float32, device=h.device)
        _native.mp("edge_pair", h, G.ef, G.src, G.dst, G.E, WIDTH, EDGE_F, R)
        s = _mm(R, p["wo"]).reshape(-1) + p["bo"]
        s = s.contiguous()
        gamma = torch.empty(G.E, dtype=torch.float64, device=h.device)
        _native.mp("softplus", s, G.E, GAMMA_FLOOR, gamma, None, None)
        c["R"], c["s"] = R, s
        return gamma, c

    def backward(self, G: BeadGraph, c, dgamma: torch.Tensor):
        """Accumulate d(loss)/d(params) into self.grad given d(loss)/d(gamma)."""
        p, g = self.p, self.g
        ds = torch.empty(G.E, dtype=torch.float32, device=dgamma.device)
        _native.mp("softplus", c["s"], G.E, GAMMA_FLOOR, None, dgamma.contiguous(), ds)
        _mm(c["R"].t(), ds[:, None], out=g["wo"], accumulate=True)
        _colsum(ds[:, None], g["bo"][None, :])
        dR = (ds[:, None] * p["wo"].reshape(1, -1)).contiguous()
        dh = torch.zeros((G.n, WIDTH), dtype=torch.float32, device=ds.device)
        _native.mp("edge_pair_bwd", dR, G.src, G.dst, G.E, WIDTH, EDGE_F, dh)
        for l in reversed(range(LAYERS)):
            Z, A, U, T = c[l]
            dT = dh.clone()
            _native.mp("relu_bwd", dT, T, dT.numel())
            _mm(U.t(), dT, out=g[f"Wu{l}"], accumulate=True)
            _colsum(dT, g[f"bu{l}"][None, :])
            dU = _mm(dT, p[f"Wu{l}"].t())
            dM = dU[:, WIDTH:].contiguous()
            dh = dh + dU[:, :WIDTH]
            dA = torch.empty((G.E, WIDTH), dtype=torch.float32, device=ds.device)
            _native.mp("segment_sum_bwd", dM, G.mp_rowptr, G.dst, G.E, WIDTH, dA)
            _native.mp("relu_bwd", dA, A, dA.numel())
            _mm(Z.t(), dA, out=g[f"Wm{l}"], accumulate=True)
            _colsum(dA, g[f"bm{l}"][None, :])
            dZ = _mm(dA, p[f"Wm{l}"].t())
            dh = dh.contiguous()
            _native.mp("edge_concat_bwd", dZ, G.src, G.E, WIDTH, EDGE_F, dh)
        _native.mp("relu_bwd", dh, c["h0"], dh.numel())
        _mm(G.x.t(), dh, out=g["W0"], accumulate=True)
        _colsum(dh, g["b0"][None, :])

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        _native.mp("adam", self.flat, self.grad, self.m1, self.m2, self.flat.numel(), lr, b1, b2, eps, self.step)
        self.grad.zero_()


# ---------------------------------------------------------------------------
# Bead model solve, loss and training
# ---------------------------------------------------------------------------
def bead_modes(G: BeadGraph, gamma_mp, m, tol=1e-8):
    """Lowest m non-rigid eigenpairs of the bead model with spring constants gamma."""
    from .solvers.chfsi import chfsi
    H = HessianStore(G.pos, G.rc_nm * 10.0, plus_i=1.0, precisions=("f64",),
                     graph_=(G.degree, G.rowptr, G.cols), pair_weight=G.adjacency_weights(gamma_mp))
    Q = rigid_body_basis(G.pos)
    ev, V = chfsi(H, m, tol=tol, Q=Q, precision="f64")
    return ev - 1.0, V


def loss_and_grad(G: BeadGraph, gamma_mp, lam_fine: torch.Tensor, reg=0.0):
    """(loss, d loss / d gamma, bead eigenvalues) for the mean squared log ratio
    of the bead model's eigenvalues to the fine ones, plus reg * mean((log gamma)^2),
    which keeps the springs near the uniform model (gamma = 1) unless moving them
    pays in eigenvalues."""
    m = lam_fine.shape[0]
    lam, V = bead_modes(G, gamma_mp, m)
    r = torch.log(lam / lam_fine)
    loss = float((r ** 2).mean())
    c = (2.0 * r / lam / m).contiguous()
    dgamma = torch.empty(G.E, dtype=torch.float64, device=gamma_mp.device)
    _native.mp("hf_grad", G.pos, G.mp_rowptr, G.src, G.dst, V.contiguous(), m, c, G.E, dgamma)
    if reg > 0.0:
        lg = torch.log(gamma_mp)
        loss += reg * float((lg ** 2).mean())
        dgamma += (2.0 * reg / G.E) * lg / gamma_mp
    return loss, dgamma, lam


def train(model: WarmStartMPNN, samples, epochs=50, lr=3e-3, verbose=True, reg=0.0):
    """samples: list of (BeadGraph, fine eigenvalues (m,) tensor).  Returns the
    per-epoch mean loss."""
    hist = []
    for ep in range(epochs):
        tot = 0.0
        for G, lam_f in samples:
            gamma, cache = model.forward(G)
            loss, dgamma, _ = loss_and_grad(G, gamma, lam_f, reg=reg)
            model.backward(G, cache, dgamma)
            model.adam(lr=lr)
            tot += loss
        hist.append(tot / len(samples))
        if verbose:
            print(f"epoch {ep}: mean loss {hist[-1]:.4e}", flush=True)
    return hist


TEST_COLUMNS = 64     # leading columns of each block that the residual test looks at


def _median_ritz_residual(H, V, k, Q):
    """Median ||H y - theta y|| over the k lowest Ritz pairs of span(V) (rigid
    modes projected out), from one FP32 SpMM of V's width."""
    from .solvers.chfsi import _cholqr, _project_out, _rr
    Y = _cholqr(_project_out(V, Q))
    th, Y, HY = _rr(H, Y, 32)
    R = HY[:, :k] - Y[:, :k] * torch.from_numpy(th[:k]).to(Y.device)[None, :]
    return float(torch.linalg.vector_norm(R, dim=0).median())


def learned_warm_start(X_nm: torch.Tensor, n_vectors: int, model: WarmStartMPNN, fine_rowptr=None, fine_cols=None,
                       bead_edge_A=6.0, rc_bead_A=12.0, tol=1e-4, H=None, Q=None, k=None, seed=0,
                       return_info=False):
    """(3N, n_vectors) FP64 initial block from the learned bead model's lowest modes.
    With k (the wanted fine modes), only the k lowest bead modes are converged and
    the rest of the block is the coarse solver's guard Ritz vectors.

    With the fine Hessian store H (and its rigid basis Q), the block must pass the
    residual test: over the leading TEST_COLUMNS columns (the lowest bead modes),
    the median residual of the Ritz pairs below that of as many random columns;
    otherwise a random block is returned.  (A test over the full width costs two
    Rayleigh-Ritz passes of the whole block: 3-4 s for 1,250 columns of 1.5M dof.)"""
    from .solvers.chfsi import chfsi
    G = BeadGraph(X_nm, fine_rowptr, fine_cols, bead_edge_A, rc_bead_A)
    gamma, _ = model.forward(G)
    m = min(n_vectors, 3 * G.n - 7)
    info = dict(beads=G.n, coarse_modes=m, fallback=False)
    gen = torch.Generator(device=X_nm.device)
    gen.manual_seed(seed)
    V = None
    if bool(torch.isfinite(gamma).all()):
        Hb = HessianStore(G.pos, rc_bead_A, plus_i=1.0, graph_=(G.degree, G.rowptr, G.cols),
                          pair_weight=G.adjacency_weights(gamma))
        kc = m if k is None else max(1, min(int(k), m))    # as in warmstart.coarse_warm_start(wanted=k)
        _, Vc = chfsi(Hb, kc, tol=tol, Q=rigid_body_basis(G.pos), precision="mixed", seed=seed + 7,
                      guard=m - kc if kc < m else None, final_f64=False, return_block=kc < m)
        V = Vc.reshape(G.n, 3, m).index_select(0, G.bead).reshape(3 * X_nm.shape[0], m)
        if m < n_vectors:
            V = torch.cat([V, torch.randn((V.shape[0], n_vectors - m), generator=gen, dtype=V.dtype,
                                          device=V.device)], dim=1)
    if H is not None:
        t = min(TEST_COLUMNS, n_vectors)
        kk = min(k if k is not None else t, t)
        Vr = torch.randn((3 * X_nm.shape[0], t), generator=gen, dtype=torch.float64, device=X_nm.device)
        info["random_median_residual"] = _median_ritz_residual(H, Vr, kk, Q)
        if V is not None:
            info["warm_median_residual"] = _median_ritz_residual(H, V[:, :t].contiguous(), kk, Q)
        if V is None or not info["warm_median_residual"] < info["random_median_residual"]:
            V = torch.randn((3 * X_nm.shape[0], n_vectors), generator=gen, dtype=torch.float64,
                            device=X_nm.device)
            info["fallback"] = True
    elif V is None:
        raise AssertionError("ABORTED. the network produced non-finite spring constants")
    return (V, info) if return_info else V


# ---------------------------------------------------------------------------
# Training data and entry point
# ---------------------------------------------------------------------------
def training_structures(n_struct=24, seed=7):
    """Seeded synthetic structures for training: single globules and touching
    assemblies of 2-8 globules, 2,000-16,000 atoms in total."""
    from . import synth
    rng = np.random.default_rng(seed)
    out = []
    for t in range(n_struct):
        if t % 2 == 0:
            n = int(np.exp(rng.uniform(np.log(2000), np.log(12000))))
            X = synth.globule(n, seed=10_000 + t)
        else:
            g = int(rng.integers(2, 9))
            size = int(rng.integers(1000, 2000))
            X = synth.touching_assembly([size] * g, seed=20_000 + t)
        out.append(X / 10.0)
    return out


def make_sample(X_nm_host, m=32, bead_edge_A=6.0, rc_bead_A=12.0):
    """(BeadGraph, lowest m non-rigid fine eigenvalues from the plain FP64 solver)."""
    from . import graph
    from .solvers.chfsi import chfsi
    Xd = torch.from_numpy(np.ascontiguousarray(X_nm_host)).cuda()
    order, _ = graph.cuthill_mckee(Xd, 8.0)
    Xr = Xd[order]
    H = HessianStore(Xr, 8.0, 1.0, precisions=("f64",))
    ev, _ = chfsi(H, m, tol=1e-9, Q=rigid_body_basis(Xr), precision="f64")
    G = BeadGraph(Xr, H.rowptr, H.cols, bead_edge_A, rc_bead_A)
    return G, (ev - 1.0).contiguous()


def main(argv=None):
    import argparse
    import time
    ap = argparse.ArgumentParser(description="train the warm-start network on synthetic structures (GPU)")
    ap.add_argument("--structures", type=int, default=24)
    ap.add_argument("--epochs", type=int, default=50)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--reg", type=float, default=0.0, help="weight of mean((log gamma)^2)")
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    samples = [make_sample(X) for X in training_structures(a.structures)]
    t1 = time.perf_counter()
    model = WarmStartMPNN()
    hist = train(model, samples, epochs=a.epochs, lr=a.lr, reg=a.reg)
    model.save(a.out, epochs=a.epochs, structures=a.structures, reg=a.reg, first_loss=hist[0], last_loss=hist[-1],
               data_seconds=t1 - t0, train_seconds=time.perf_counter() - t1)
    print(f"saved {a.out}: loss {hist[0]:.4e} -> {hist[-1]:.4e}")


if __name__ == "__main__":
    main()
