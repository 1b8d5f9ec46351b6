"""Autotuner host logic on CPU: the fastest candidate is applied and remembered
on the store, the choice is cached per (atoms, pairs, width class, precision,
device), the band-tile layout is tried only when the store has tiles, and the
launch hooks of the C ABI accept the documented settings and reject others (no
GPU call is involved)."""
import pytest
import torch

COST = {("pairs", 256, 5, 1): 3.0, ("pairs", 256, 5, 0): 2.2, ("pairs", 256, 5, 2): 2.9,
        ("pairs", 256, 4, 1): 2.0, ("pairs", 512, 2, 1): 2.5, ("pairs", 0, 4, 0): 1.5,
        ("groups", 256, 5, 1): 1.2, ("tiles", 256, 5, 1): 1.0}


class FakeStore:
    def __init__(self, tiles, groups=False):
        self.n_atoms, self.nnz_blocks = 100, 900
        self.shape = (300, 300)
        self.device = torch.device("cpu")
        self.tiles = {} if tiles else None
        self.use_tiles = False
        self.groups = {} if groups else None
        self.use_groups = False
        self.keep_pairs = True
        self.spmm_cfg = {}
        self.calls = 0

    def matmul(self, X, out=None, prec=32):
        self.calls += 1
        self.last_prec = prec
        out.copy_(X)
        return out


def test_autotuner_picks_fastest_and_caches(monkeypatch):
    from inching_b200 import autotune
    applied = [(256, 5, 1)]
    monkeypatch.setattr(autotune._native, "spmm_tune", lambda t, b, tr=None: applied.append((t, b, tr)))
    autotune._cache.clear()
    timed = []

    def timer(fn, reps):
        fn()
        if H.use_tiles:
            cfg = ("tiles", 256, 5, 1)
        elif H.use_groups and H.last_prec == 32:      # the row groups hold FP32 entries only
            cfg = ("groups",) + applied[-1]
        else:
            cfg = ("pairs",) + applied[-1]
        timed.append(cfg)
        return COST[cfg]

    H = FakeStore(tiles=False)
    best, table = autotune.tune_spmm(H, 64, timer=timer)
    assert best == ("pairs", 0, 4, 0) and applied[-1] == (0, 4, 0) and not H.use_tiles
    assert H.spmm_cfg[(32, 64)] == best
    assert set(table) == {c for c in COST if c[0] == "pairs"} and len(timed) == 6 and H.calls == 6
    again = autotune.tune_spmm(H, 100, timer=timer)          # same width class (64): cached
    assert again[0] == best and len(timed) == 6 and applied[-1] == (0, 4, 0)
    autotune.tune_spmm(H, 16, timer=timer)                   # another width class: timed again
    assert len(timed) == 12 and (32, 8) in H.spmm_cfg
    H = FakeStore(tiles=True)
    H.nnz_blocks = 901                                       # another store
    best, table = autotune.tune_spmm(H, 64, timer=timer)
    assert best == ("tiles", 256, 5, 1) and H.use_tiles and len(table) == 7
    assert H.spmm_cfg[(32, 64)] == best
    # the row-group layout: timed for FP32 products of >= 64 columns when built
    H = FakeStore(tiles=False, groups=True)
    H.nnz_blocks = 902
    best, table = autotune.tune_spmm(H, 128, timer=timer)
    assert best == ("groups", 256, 5, 1) and H.use_groups and not H.use_tiles and len(table) == 7
    autotune.apply_config(H, ("pairs", 256, 5, 1))
    assert not H.use_groups
    H.nnz_blocks = 903
    best, table = autotune.tune_spmm(H, 32, timer=timer)     # narrower than one group tile
    assert ("groups", 256, 5, 1) not in table and best == ("pairs", 0, 4, 0)
    H.nnz_blocks = 904
    H.use_groups = True
    best, table = autotune.tune_spmm(H, 64, prec=64, timer=timer)   # FP64: pair layout only
    assert ("groups", 256, 5, 1) not in table
    assert H.use_groups                     # an FP64 choice leaves the FP32 layout alone
    autotune._cache.clear()


def test_layout_pinned_by_environment(monkeypatch):
    """INCH_SPMM_LAYOUT restricts the candidates to one layout where the store has
    it, and is ignored where it has not."""
    from inching_b200 import autotune
    monkeypatch.setattr(autotune._native, "spmm_tune", lambda t, b, tr=None: None)
    autotune._cache.clear()
    monkeypatch.setenv("INCH_SPMM_LAYOUT", "pairs")
    H = FakeStore(tiles=False, groups=True)
    best, table = autotune.tune_spmm(H, 128, timer=lambda fn, reps: (fn(), 1.0)[1])
    assert {c[0] for c in table} == {"pairs"} and not H.use_groups
    monkeypatch.setenv("INCH_SPMM_LAYOUT", "groups")
    H = FakeStore(tiles=False, groups=True)
    H.nnz_blocks = 905
    best, table = autotune.tune_spmm(H, 128, timer=lambda fn, reps: (fn(), 1.0)[1])
    assert best[0] == "groups" and len(table) == 1 and H.use_groups
    H.nnz_blocks = 906
    best, table = autotune.tune_spmm(H, 64, prec=64, timer=lambda fn, reps: (fn(), 1.0)[1])
    assert {c[0] for c in table} == {"pairs"}          # no FP64 groups: the pin is ignored
    autotune._cache.clear()


def test_launch_hooks_accept_documented_settings_only():
    from inching_b200 import _native, autotune
    for t, b in ((256, 5), (512, 2), (1024, 1), (0, 4)):
        for tr in (0, 1, 2):
            _native.spmm_tune(t, b, tr)
    with pytest.raises(AssertionError):
        _native.spmm_tune(300, 5)
    with pytest.raises(AssertionError):
        _native.spmm_tune(256, 5, 3)
    _native.spmm_band_tune(64)
    _native.spmm_band_tune(128)
    for u in (0, 2, 4, 8, 16):
        _native.spmm_group_tune(u)
    with pytest.raises(AssertionError):
        _native.spmm_group_tune(3)
    with pytest.raises(AssertionError):
        _native.spmm_band_tune(96)
    autotune.reset()
    assert autotune._cache == {}
