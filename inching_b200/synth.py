"""Seeded synthetic macromolecular structures (coordinates in Angstrom).

The reference benchmarks real PDB/CIF assemblies that are not available here, so
these generators stand in for them with matching atom counts and neighbour
densities (about 120 atoms within 8 A at 0.056 atoms/A^3 in the bulk).

Construction of one globule of N atoms:
  * the globule is a ball of radius R = (3N / (4 pi rho))^(1/3), rho = 0.056 A^-3;
  * atoms sit on a cubic lattice of spacing a = rho^(-1/3) (2.61 A) clipped to the
    ball (the N sites closest to the centre are kept), each displaced by a
    seeded uniform jitter of +-0.3 a per axis, so no two atoms coincide and no
    pair sits exactly on the cutoff;
  * atoms are numbered along a 3-D Hilbert curve through the lattice, i.e. the
    chain is a compact self-avoiding walk whose consecutive atoms are
    neighbours, as sequence-local as a protein chain in PDB order.

Assemblies place globules so that neighbouring surfaces touch; atom numbering
runs globule after globule, as chains do in a multi-chain PDB file.
"""
from __future__ import annotations

import numpy as np

RHO = 0.056          # atoms per A^3
JITTER = 0.3         # fraction of the lattice spacing


def globule_radius(n_atoms: int, rho: float = RHO) -> float:
    return float((3.0 * n_atoms / (4.0 * np.pi * rho)) ** (1.0 / 3.0))


def _hilbert_index(coords: np.ndarray, bits: int) -> np.ndarray:
    """Hilbert-curve index of non-negative integer points (M, 3), Skilling's
    transpose algorithm (AIP Conf. Proc. 707, 381 (2004)), vectorised."""
    x = coords.astype(np.int64).T.copy()          # (3, M)
    n = 3
    m = 1 << (bits - 1)
    # inverse undo excess work
    q = m
    while q > 1:
        p = q - 1
        for i in range(n):
            hit = (x[i] & q) != 0
            # invert low bits of x[0] where hit
            x[0] = np.where(hit, x[0] ^ p, x[0])
            # exchange low bits of x[0] and x[i] where not hit
            t = (x[0] ^ x[i]) & p
            t = np.where(hit, 0, t)
            x[0] ^= t
            x[i] ^= t
        q >>= 1
    # Gray encode
    for i in range(1, n):
        x[i] ^= x[i - 1]
    t = np.zeros_like(x[0])
    q = m
    while q > 1:
        t = np.where((x[n - 1] & q) != 0, t ^ (q - 1), t)
        q >>= 1
    for i in range(n):
        x[i] ^= t
    # interleave transposed bits into one index (x[0] holds the top bit)
    h = np.zeros(x.shape[1], dtype=np.int64)
    for b in range(bits - 1, -1, -1):
        for i in range(n):
            h = (h << 1) | ((x[i] >> b) & 1)
    return h


def globule(n_atoms: int, seed: int, rho: float = RHO) -> np.ndarray:
    """One compact globule of ``n_atoms`` atoms centred at the origin (float64, A)."""
    if n_atoms <= 0:
        return np.zeros((0, 3), dtype=np.float64)
    rng = np.random.default_rng(seed)
    a = rho ** (-1.0 / 3.0)
    R = globule_radius(n_atoms, rho)
    half = int(np.ceil(R / a)) + 2
    g = np.arange(-half, half + 1)
    ii, jj, kk = np.meshgrid(g, g, g, indexing="ij")
    sites = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
    # random sub-lattice offset so that globules are not all identical
    off = rng.uniform(-0.5, 0.5, size=3)
    r2 = ((sites + off) ** 2).sum(axis=1)
    keep = np.argsort(r2, kind="stable")[:n_atoms]
    sites = sites[keep]
    bits = int(np.ceil(np.log2(2 * half + 2)))
    h = _hilbert_index(sites + half, bits)
    sites = sites[np.argsort(h, kind="stable")]
    X = (sites + off) * a + rng.uniform(-JITTER, JITTER, size=(n_atoms, 3)) * a
    X -= X.mean(axis=0)
    return X.astype(np.float64)


def touching_assembly(sizes, seed: int, rho: float = RHO) -> np.ndarray:
    """Globules of the given sizes whose centres lie on a simple-cubic grid with
    spacing equal to the largest diameter, so that neighbouring spheres touch.
    The grid sites nearest the grid centre are used."""
    sizes = [int(s) for s in sizes]
    n = len(sizes)
    side = int(np.ceil(n ** (1.0 / 3.0)))
    g = np.arange(side)
    ii, jj, kk = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    pts -= pts.mean(axis=0)
    order = np.argsort((pts ** 2).sum(axis=1), kind="stable")[:n]
    pts = pts[order]
    spacing = 2.0 * max(globule_radius(s, rho) for s in sizes)
    parts = []
    for t, s in enumerate(sizes):
        parts.append(globule(s, seed * 1000003 + t, rho) + pts[t] * spacing)
    X = np.concatenate(parts, axis=0)
    return X - X.mean(axis=0)


def shell_assembly(n_sub: int, sub_atoms: int, radius: float, seed: int,
                   rho: float = RHO) -> np.ndarray:
    """``n_sub`` globules centred on a Fibonacci lattice of a sphere of ``radius``."""
    k = np.arange(n_sub) + 0.5
    phi = np.arccos(1 - 2 * k / n_sub)
    theta = np.pi * (1 + 5 ** 0.5) * k
    centres = radius * np.stack([np.cos(theta) * np.sin(phi),
                                 np.sin(theta) * np.sin(phi), np.cos(phi)], axis=1)
    parts = [globule(sub_atoms, seed * 1000003 + t, rho) + centres[t] for t in range(n_sub)]
    return np.concatenate(parts, axis=0)


def batch_sizes(n_struct: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """Structure sizes drawn log-uniform over [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_struct)).astype(np.int64)


# Named workloads (atom counts and layouts of the benchmark configurations).
def workload(name: str) -> np.ndarray:
    if name == "globule5k":            # one globule, 5,000 atoms
        return globule(5000, seed=0)
    if name == "assembly100k":         # 20 touching globules of 5,000 atoms
        return touching_assembly([5000] * 20, seed=1)
    if name == "shell500k":            # 60 subunits of ~8,300 atoms on a 250 A sphere
        return shell_assembly(60, 8300, 250.0, seed=3)
    if name == "cube2400k":            # ~300 touching globules of ~8,000 atoms
        return touching_assembly([8000] * 300, seed=4)
    raise KeyError(name)
