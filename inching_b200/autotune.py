"""Autotuner for the wide-block Hessian products (no reference counterpart).

For a given store, block width and precision it times the candidate launch
configurations of the SpMM with CUDA events on the current stream and keeps the
fastest, for the process and on the store itself (the store re-applies its own
choice before each product, so stores of different sizes keep their own):
  * layout: the pair layout (one entry per neighbour pair), the row-group layout
    (FP32; 2 consecutive rows merged over their neighbour lists, one gather of X_j
    for both), when the store has it, or the band-tile layout (8-row tiles with
    merged neighbour unions), when the store has tiles;
  * lane-group kernel block shape: 256 x 5, 256 x 4, 512 x 2 blocks/SM;
  * row traversal of the lane-group kernel: fixed grid stride (the warps of a
    block on neighbouring rows share their X_j rows in L1), or chunks of rows
    from a counter per warp or per block (one compact frontier over all SMs keeps
    the X_j rows in L2 on large structures);
  * the whole-warp-row kernel with batched gathers ("pairs", 0, ...).
Results are cached per (atoms, pairs, width class, precision, device name).
The solvers call tune_spmm once per store for the widths they use.  The
environment variable INCH_SPMM_LAYOUT (pairs, groups or tiles) restricts the
candidates to one layout where the store has it (to pin the layout of a run, e.g.
for a profile whose own timing would distort the comparison).
"""
from __future__ import annotations

import os

import torch

from . import _native

# (layout, threads per block (0: whole-warp kernel), blocks per SM, traversal)
CANDIDATES = (("pairs", 256, 5, 1), ("pairs", 256, 5, 0), ("pairs", 256, 5, 2), ("pairs", 256, 4, 1),
              ("pairs", 512, 2, 1), ("pairs", 0, 4, 0), ("groups", 256, 5, 1), ("tiles", 256, 5, 1))
_cache = {}


def _width_class(b):
    from .hessian import width_class
    return width_class(b)


def _apply(H, cfg, prec=32):
    apply_config(H, cfg, prec)


def apply_config(H, cfg, prec=32):
    """Make cfg = (layout, threads, blocks per SM, traversal) the current choice for
    products at precision prec.  The row-group layout holds FP32 entries only, so
    only an FP32 choice switches it on or off."""
    layout, threads, bps, trav = cfg
    if layout in ("pairs", "groups"):
        _native.spmm_tune(threads, bps, trav)
    H.use_tiles = layout == "tiles"
    if getattr(H, "groups", None) is not None and prec == 32:
        H.use_groups = layout == "groups"


def cuda_event_ms(fn, reps):
    """Fastest of `reps` runs of fn in ms, CUDA events on the current stream, after
    one untimed run."""
    fn()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for e0, e1 in ev:
        e0.record()
        fn()
        e1.record()
    torch.cuda.synchronize()
    return min(e0.elapsed_time(e1) for e0, e1 in ev)


def _device_name(dev):
    dev = torch.device(dev)
    return torch.cuda.get_device_name(dev) if dev.type == "cuda" else dev.type


def tune_spmm(H, b, prec=32, reps=5, candidates=CANDIDATES, timer=cuda_event_ms):
    """Pick and apply the fastest configuration for (H, b, prec); returns (cfg, ms
    table).  timer(fn, reps) -> ms measures one candidate."""
    key = (H.n_atoms, H.nnz_blocks, _width_class(b), prec, _device_name(H.device))
    if key in _cache:
        _apply(H, _cache[key][0], prec)
        _remember(H, prec, b, _cache[key][0])
        return _cache[key]
    dt = torch.float64 if prec == 64 else torch.float32
    w = _width_class(b) if b >= 8 else b
    forced = os.environ.get("INCH_SPMM_LAYOUT")
    if forced:
        pinned = tuple(c for c in candidates if c[0] == forced and _available(H, c, prec, w))
        candidates = pinned or candidates
    X = torch.randn((H.shape[0], w), dtype=dt, device=H.device)
    Y = torch.empty_like(X)
    table = {}
    for cfg in candidates:
        if not _available(H, cfg, prec, w):
            continue
        _apply(H, cfg, prec)
        table[cfg] = timer(lambda: H.matmul(X, out=Y, prec=prec), reps)
    best = min(table, key=table.get)
    _apply(H, best, prec)
    _remember(H, prec, b, best)
    _cache[key] = (best, table)
    return best, table


def _available(H, cfg, prec, w):
    """Whether the store can run candidate cfg for a w-column product at prec."""
    if cfg[0] == "tiles":
        return H.tiles is not None
    if cfg[0] == "groups":
        return getattr(H, "groups", None) is not None and prec == 32 and w >= 64
    return H.keep_pairs


def _remember(H, prec, b, cfg):
    cfgs = getattr(H, "spmm_cfg", None)
    if cfgs is not None:
        cfgs[(prec, _width_class(b))] = cfg


def reset():
    """Forget the cached choices and restore the default launch shape (256 x 5,
    pair layout kernel, per-warp row chunks)."""
    _cache.clear()
    _native.spmm_tune(256, 5, 1)
