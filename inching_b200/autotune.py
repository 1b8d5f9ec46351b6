"""Autotuner for the wide-block Hessian products (no reference counterpart).

For a given store, block width and precision it times the candidate launch
configurations of the SpMM with CUDA events on the current stream and keeps the
fastest for the process:
  * layout: the pair layout (one entry per neighbour pair) or the row-tile layout
    (8-row tiles with merged neighbour unions), when the store has tiles;
  * lane-group kernel block shape: 256 x 5, 256 x 4, 512 x 2, 1024 x 1 blocks/SM;
  * the whole-warp-row kernel with batched gathers ("warp", for >= 32 columns).
Results are cached per (atoms, pairs, width class, precision, device name).
"""
from __future__ import annotations

import torch

from . import _native

CANDIDATES = (("pairs", 256, 5), ("pairs", 256, 4), ("pairs", 512, 2), ("pairs", 1024, 1), ("pairs", 0, 4),
              ("tiles", 256, 5))
_cache = {}


def _width_class(b):
    return 64 if b >= 64 else (32 if b >= 32 else (8 if b >= 8 else b))


def _apply(H, cfg):
    layout, threads, bps = cfg
    _native.spmm_tune(threads, bps)
    H.use_tiles = layout == "tiles"


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


def tune_spmm(H, b, prec=32, reps=3, candidates=CANDIDATES, timer=cuda_event_ms):
    """Pick and apply the fastest configuration for (H, b, prec); returns (cfg, ms
    table).  timer(fn, reps) -> ms measures one candidate."""
    key = (H.n_atoms, H.nnz_blocks, _width_class(b), prec, _device_name(H.device))
    if key in _cache:
        _apply(H, _cache[key][0])
        return _cache[key]
    dt = torch.float64 if prec == 64 else torch.float32
    w = _width_class(b) if b >= 8 else b
    X = torch.randn((H.shape[0], w), dtype=dt, device=H.device)
    Y = torch.empty_like(X)
    table = {}
    for cfg in candidates:
        if cfg[0] == "tiles" and H.tiles is None:
            continue
        _apply(H, cfg)
        table[cfg] = timer(lambda: H.matmul(X, out=Y, prec=prec), reps)
    best = min(table, key=table.get)
    _apply(H, best)
    _cache[key] = (best, table)
    return best, table


def reset():
    """Forget the cached choices and restore the default launch shape (256 x 5,
    pair layout kernel)."""
    _cache.clear()
    _native.spmm_tune(256, 5)
