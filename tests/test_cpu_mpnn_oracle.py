"""The message-passing network oracle checked against finite differences, and
the Hellmann-Feynman eigenvalue gradient of the bead Hessian against finite
differences of dense eigenvalues (CPU, FP64)."""
import numpy as np

from oracle import mpnn


def _graph(rng, n=7):
    pos = rng.standard_normal((n, 3))
    src, dst = [], []
    for a in range(n):
        for b in range(n):
            if a != b and np.linalg.norm(pos[a] - pos[b]) < 1.8:
                dst.append(a)
                src.append(b)
    return pos, np.array(src), np.array(dst)


def _params(rng, W=6, F=4, G=4, layers=3):
    p = {"W0": rng.standard_normal((F, W)) * 0.5, "b0": rng.standard_normal(W) * 0.1}
    for l in range(layers):
        p[f"Wm{l}"] = rng.standard_normal((W + G, W)) * 0.4
        p[f"bm{l}"] = rng.standard_normal(W) * 0.1
        p[f"Wu{l}"] = rng.standard_normal((2 * W, W)) * 0.4
        p[f"bu{l}"] = rng.standard_normal(W) * 0.1
    p["wo"] = rng.standard_normal((W + G, 1)) * 0.3
    p["bo"] = np.array([0.2])
    return p


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    pos, src, dst = _graph(rng)
    x = rng.standard_normal((len(pos), 4))
    ef = rng.standard_normal((len(src), 4))
    p = _params(rng)
    w = rng.standard_normal(len(src))
    gam, c = mpnn.forward(p, x, ef, src, dst, len(pos))
    g = mpnn.backward(p, x, ef, src, dst, len(pos), c, w)
    for name in ("W0", "Wm1", "Wu2", "wo", "bm0", "bo"):
        flat = p[name].reshape(-1)
        for idx in rng.choice(flat.size, size=min(4, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + 1e-6
            fp = w @ mpnn.forward(p, x, ef, src, dst, len(pos))[0]
            flat[idx] = old - 1e-6
            fm = w @ mpnn.forward(p, x, ef, src, dst, len(pos))[0]
            flat[idx] = old
            fd = (fp - fm) / 2e-6
            assert abs(fd - g[name].reshape(-1)[idx]) <= 1e-5 * max(1.0, abs(fd)), name


def test_hellmann_feynman_matches_finite_differences():
    rng = np.random.default_rng(1)
    pos, src, dst = _graph(rng, n=8)
    # symmetric constants per pair
    gam = np.empty(len(src))
    for e in range(len(src)):
        gam[e] = 1.0 + 0.3 * np.sin(min(src[e], dst[e]) + 2 * max(src[e], dst[e]))
    H = mpnn.bead_hessian(pos, src, dst, gam)
    w, V = np.linalg.eigh(H)
    c = rng.standard_normal(6)
    sel = slice(6, 12)           # lowest non-rigid eigenpairs (rigid ones sit at PlusI)
    g = mpnn.hf_grad(pos, src, dst, V[:, sel], c)
    # perturb one pair (both directions), compare with d/dgamma of sum c_t lambda_t
    e = 0
    pair = [i for i in range(len(src)) if {src[i], dst[i]} == {src[e], dst[e]}]
    h = 1e-6
    gp = gam.copy()
    gp[pair] += h
    wp = np.linalg.eigvalsh(mpnn.bead_hessian(pos, src, dst, gp))
    gm = gam.copy()
    gm[pair] -= h
    wm = np.linalg.eigvalsh(mpnn.bead_hessian(pos, src, dst, gm))
    fd = c @ (wp[sel] - wm[sel]) / (2 * h)
    assert abs(fd - g[pair].sum()) <= 1e-5 * max(1.0, abs(fd))
