"""The block-banded ANM Hessian store and its operator.

`HessianStore` stands where the reference returns its lower-triangle CuPy CSR
matrix (InchingLiteInteger/Fuel/T1.py:655-660): it has ``shape``, ``dtype`` and
``ndim`` (the solvers' argument checks read them, e.g. ThickRestartLanczos.../
T1.py:85-87) and holds, on the GPU, the Cuthill-McKee-banded adjacency and the
rank-one block store (w = x/|x| per pair, symmetric diagonal blocks) in FP64
and/or FP32.  Products go through the fused SpMM kernel.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native, graph

# Optional recorder of SpMM calls (CUDA events + algorithmic bytes); set by
# measurement code, None otherwise.
_probe = None


class SpmmProbe:
    """Records, for every store product issued while active, start/end CUDA events
    on the launching (current) stream and the call's algorithmic bytes:
    store once + X read once + Y written once (+ Yin / Acc traffic)."""

    def __init__(self, prec=None):
        self.prec = prec
        self.records = []

    def __enter__(self):
        global _probe
        _probe = self
        return self

    def __exit__(self, *a):
        global _probe
        _probe = None

    def summary(self):
        torch.cuda.synchronize()
        ms = sum(s.elapsed_time(e) for s, e, _, _ in self.records)
        nbytes = sum(b for _, _, b, _ in self.records)
        calls = len(self.records)
        return dict(calls=calls, ms=ms, bytes=nbytes, launches=sum(l for *_, l in self.records))


class HessianStore:
    """ANM Hessian H + PlusI*I of a structure whose atoms are already in the
    order the caller wants (normally reversed Cuthill-McKee)."""

    def __init__(self, X_nm, rc_gamma_A: float = 8.0, plus_i: float = 1.0, precisions=("f64", "f32"),
                 device=None, graph_=None, tiles=False, pair_weight=None, pbc=None, keep_pairs=True,
                 groups=2):
        self.X = graph.to_device_coords(X_nm, device)
        self.device = self.X.device
        self.n_atoms = int(self.X.shape[0])
        self.rc_nm = rc_gamma_A / 10.0
        self.plus_i = float(plus_i)
        self.box_xy = graph.pbc_box(pbc)     # periodic xy images (nm) or None
        if graph_ is None:
            graph_ = _native.neighbor_lists(self.X, self.rc_nm, box_xy=self.box_xy)
        self.degree, self.rowptr, self.cols = graph_[:3]
        self.image = graph_[3] if len(graph_) > 3 else None
        if (self.box_xy is None) != (self.image is None):
            raise AssertionError("ABORTED. periodic images need both the box and the image codes of the lists")
        if tiles == "auto":
            # the band-tile layout takes neither periodic images nor per-pair springs
            tiles = self.box_xy is None and pair_weight is None and self.n_atoms < (1 << 24)
        # The band tiles are an opt-in layout: on the B200 the pair kernel's wide
        # product is faster (0.52 ms against 1.05 ms for 64 columns of the 100k-atom
        # assembly), so products use the band tiles only when they are built.
        if self.box_xy is not None and tiles:
            raise AssertionError("ABORTED. the row-tile layout does not take periodic images")
        if pair_weight is not None and tiles:
            raise AssertionError("ABORTED. the row-tile layout does not take per-pair spring constants")
        if not keep_pairs and not tiles:
            raise AssertionError("ABORTED. keep_pairs=False needs the row-tile layout")
        want64 = "f64" in precisions
        want32 = "f32" in precisions
        self.ent64, self.diag64, self.ent32, self.diag32 = _native.hessian_assemble(
            self.X, self.rowptr, self.cols, self.rc_nm, self.plus_i, want64, want32, pair_weight=pair_weight,
            image=self.image, box_xy=self.box_xy)
        n = 3 * self.n_atoms
        self.shape = (n, n)
        self.ndim = 2
        self.dtype = np.dtype(np.float64)
        self.nnz_blocks = int(self.cols.shape[0])
        self._diag_vec = None
        # Row-tile layout of the same matrix for products with >= 8 columns.
        self.tiles = None
        self.use_tiles = bool(tiles)
        if tiles:
            uptr, pptr, urec, pw64, pw32, nu, npairs = _native.tile_store(self.X, self.rowptr, self.cols,
                                                                          self.rc_nm, want64, want32)
            self.tiles = dict(uptr=uptr, pptr=pptr, urec=urec, pw64=pw64, pw32=pw32, n_union=nu, n_pairs=npairs)
            if not keep_pairs:
                # every product goes through the band tiles; the pair entries are freed
                # (the diagonal blocks stay: both layouts use them)
                self.ent64 = None if self.ent64 is None else self.ent64[:0]
                self.ent32 = None if self.ent32 is None else self.ent32[:0]
        self.keep_pairs = bool(keep_pairs)
        # Row-group layout of the FP32 entries (groups = 2 or 4 consecutive rows
        # merged over their neighbour lists; 0/None: not built).  FP32 products of
        # >= 64 columns use it: each X_j gather serves every row of the group, and
        # the product gives the bits of the pair kernel (100k-atom assembly, 128
        # columns: 0.68 ms against 0.87 ms for the pair kernel).
        self.groups = None
        self.use_groups = False
        if groups and self.ent32 is not None and self.ent32.numel() > 0:
            gptr, gent, nu = _native.group_store(self.rowptr, self.ent32, self.n_atoms, int(groups))
            self.groups = dict(gptr=gptr, gent=gent, n_union=nu, rows=int(groups))
            self.use_groups = not self.use_tiles     # an explicit band-tile choice stays the default
        # autotuned launch choice per (precision, width class), set by autotune.tune_spmm
        self.spmm_cfg = {}

    # -- reference-compatible views ------------------------------------------------
    @property
    def A_diag(self) -> torch.Tensor:
        """Diagonal of H + PlusI*I, (3N,) float64 (what the reference returns beside A)."""
        if self._diag_vec is None:
            d = self.diag64 if self.diag64 is not None else self.diag32.double()
            self._diag_vec = d[:, :3].reshape(-1).contiguous()
        return self._diag_vec

    def has(self, prec: int) -> bool:
        return (self.ent64 if prec == 64 else self.ent32) is not None

    def store(self, prec: int):
        if prec == 64:
            if self.ent64 is None:
                raise AssertionError("ABORTED. the FP64 store was not assembled")
            return self.ent64, self.diag64
        if self.ent32 is None:
            raise AssertionError("ABORTED. the FP32 store was not assembled")
        return self.ent32, self.diag32

    def store_bytes(self, prec: int, b: int = 1) -> int:
        """Bytes one SpMM pass streams from the store for a b-column product: the
        row-tile layout for b >= 8 when built (records + w + offsets + diagonal),
        else the pair layout (entries + diagonal + rowptr)."""
        ent, diag = self.store(prec)
        dbytes = diag.numel() * diag.element_size()
        if self._tiled(prec, b):
            t = self.tiles
            pw = t["pw64"] if prec == 64 else t["pw32"]
            return (t["n_union"] * 4 + t["n_pairs"] * pw.shape[1] * pw.element_size()
                    + 16 * (t["uptr"].numel()) + dbytes)
        return ent.numel() * ent.element_size() + dbytes + 8 * (self.n_atoms + 1)

    # -- products ---------------------------------------------------------------
    def matmul(self, X, out=None, prec=None, **epilogue):
        """out = H X (+ fused epilogue, see _native.spmm).  prec defaults to X's dtype."""
        if prec is None:
            prec = 64 if X.dtype == torch.float64 else 32
        want = torch.float64 if prec == 64 else torch.float32
        if X.dtype != want:
            raise AssertionError(f"ABORTED. prec {prec} needs {want} vectors, got {X.dtype}")
        if (not self._tiled(prec, 1 if X.dim() == 1 else X.shape[1]) and X.dim() == 2 and X.shape[1] >= 8
                and X.shape[1] % 8 != 0 and epilogue.get("Yin") is None and epilogue.get("acc") is None):
            # pad the block to a multiple of 8 columns so every column tile runs the
            # vector-gather kernel on aligned rows; the zero columns cost < 8 columns
            b = X.shape[1]
            bp = (b + 7) // 8 * 8
            Xp = torch.zeros((X.shape[0], bp), dtype=X.dtype, device=X.device)
            Xp[:, :b] = X
            Yp = self.matmul(Xp, prec=prec, **epilogue)
            if out is None:
                return Yp[:, :b].contiguous()
            out.copy_(Yp[:, :b])
            return out
        if out is None:
            out = torch.empty_like(X)
        if self.spmm_cfg:
            cfg = self.spmm_cfg.get((prec, width_class(1 if X.dim() == 1 else X.shape[1])))
            if cfg is not None:
                from .autotune import apply_config
                apply_config(self, cfg, prec)
        ent, diag = self.store(prec)
        probe = _probe if (_probe is not None and (_probe.prec is None or _probe.prec == prec)) else None
        if probe is not None:
            b = 1 if X.dim() == 1 else X.shape[1]
            vec = X.element_size() * X.shape[0] * b
            nbytes = self.store_bytes(prec, b) + vec * (2 + (epilogue.get("Yin") is not None)
                                                     + 2 * (epilogue.get("acc") is not None))
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record()
            out = self._matmul(prec, ent, diag, X, out, epilogue)
            ev1.record()
            if self._tiled(prec, b):
                nl = _native.band_panels(prec, b)
            elif self._grouped(prec, b):
                nl = _native.group_tiles(b // 64 * 64) + _launches(b % 64, prec)
            else:
                nl = _launches(b, prec)
            probe.records.append((ev0, ev1, nbytes, nl))
            return out
        return self._matmul(prec, ent, diag, X, out, epilogue)

    def _tiled(self, prec, b):
        """Whether a b-column product at this precision runs on the band tiles: always
        when the pair entries were dropped, else for b >= 8 (narrower products keep
        the pair kernel, whose lanes split a row's entries)."""
        if self.tiles is None or not self.use_tiles:
            return False
        if (self.tiles["pw64"] if prec == 64 else self.tiles["pw32"]) is None:
            return False
        return b >= 8 or not self.keep_pairs

    def _grouped(self, prec, b):
        """Whether a b-column product runs (its first b // 64 * 64 columns) on the
        row-group layout: FP32, b >= 64, the layout built and selected."""
        return prec == 32 and b >= 64 and self.use_groups and self.groups is not None

    def _matmul(self, prec, ent, diag, X, out, epilogue):
        b = 1 if X.dim() == 1 else X.shape[1]
        if X.dim() == 2 and self._grouped(prec, b):
            G = self.groups
            bm = b // 64 * 64
            kw = dict(epilogue)
            if bm < b:
                for key in ("Yin", "acc"):
                    if kw.get(key) is not None:
                        kw[key] = kw[key][:, :bm]
            _native.spmm_groups(self.n_atoms, G["rows"], G["gptr"], G["gent"], diag, X[:, :bm], out[:, :bm], **kw)
            if bm < b:
                kw = dict(epilogue)
                for key in ("Yin", "acc"):
                    if kw.get(key) is not None:
                        kw[key] = kw[key][:, bm:]
                _native.spmm(prec, self.n_atoms, self.rowptr, ent, diag, X[:, bm:], out[:, bm:], **kw)
            return out
        if self._tiled(prec, b):
            t = self.tiles
            pw = t["pw64"] if prec == 64 else t["pw32"]
            vec = 4 if prec == 32 else 2
            X2 = X[:, None] if X.dim() == 1 else X
            out2 = out[:, None] if out.dim() == 1 else out
            kw = {k: (v[:, None] if (k in ("Yin", "acc") and v is not None and v.dim() == 1) else v)
                  for k, v in epilogue.items()}
            blocks = [X2, out2] + [kw[k] for k in ("Yin", "acc") if kw.get(k) is not None]
            if all(_band_aligned(m, vec) for m in blocks):
                _native.spmm_tiles(prec, self.n_atoms, t["uptr"], t["pptr"], t["urec"], pw, diag, X2, out2, **kw)
                return out
            # the band kernel stages 16-byte rows: run on padded copies of the blocks
            bp = (b + vec - 1) // vec * vec
            pad = lambda m: torch.nn.functional.pad(m, (0, bp - b)).contiguous()
            kwp = dict(kw)
            for k in ("Yin", "acc"):
                if kw.get(k) is not None:
                    kwp[k] = pad(kw[k])
            outp = torch.empty((X2.shape[0], bp), dtype=X2.dtype, device=X2.device)
            _native.spmm_tiles(prec, self.n_atoms, t["uptr"], t["pptr"], t["urec"], pw, diag, pad(X2), outp, **kwp)
            out2.copy_(outp[:, :b])
            if kw.get("acc") is not None:
                kw["acc"].copy_(kwp["acc"][:, :b])
            return out
        panel = 128 if prec == 32 else 64       # widest call the pair kernel takes
        if X.dim() == 1 or X.shape[1] <= panel:
            return _native.spmm(prec, self.n_atoms, self.rowptr, ent, diag, X, out, **epilogue)
        # walk column panels
        for c0 in range(0, X.shape[1], panel):
            sl = slice(c0, min(c0 + panel, X.shape[1]))
            kw = dict(epilogue)
            for key in ("Yin", "acc"):
                if kw.get(key) is not None:
                    kw[key] = kw[key][:, sl]
            _native.spmm(prec, self.n_atoms, self.rowptr, ent, diag, X[:, sl], out[:, sl], **kw)
        return out

    def matmul_seg(self, X, out, atom_seg, seg_coef, Yin=None, prec=32):
        """out = alpha_s (H X) + gamma_s X + beta_s Yin with per-segment coefficients
        (block-diagonal stores of many structures; pair layout)."""
        ent, diag = self.store(prec)
        vec = 4 if prec == 32 else 2
        b = X.shape[1]
        if self._grouped(prec, b):
            G = self.groups
            bm = b // 64 * 64
            _native.spmm_groups_seg(self.n_atoms, G["rows"], G["gptr"], G["gent"], diag, X[:, :bm], out[:, :bm],
                                    atom_seg, seg_coef, Yin=None if Yin is None else Yin[:, :bm])
            if bm < b:
                _native.spmm_seg(prec, self.n_atoms, self.rowptr, ent, diag, X[:, bm:], out[:, bm:], atom_seg,
                                 seg_coef, Yin=None if Yin is None else Yin[:, bm:])
            return out
        if self._tiled(prec, X.shape[1]) and all(_band_aligned(m, vec) for m in (X, out, Yin) if m is not None):
            t = self.tiles
            pw = t["pw64"] if prec == 64 else t["pw32"]
            return _native.spmm_tiles_seg(prec, self.n_atoms, t["uptr"], t["pptr"], t["urec"], pw, diag, X, out,
                                          atom_seg, seg_coef, Yin=Yin)
        panel = 128 if prec == 32 else 64
        for c0 in range(0, X.shape[1], panel):
            sl = slice(c0, min(c0 + panel, X.shape[1]))
            _native.spmm_seg(prec, self.n_atoms, self.rowptr, ent, diag, X[:, sl], out[:, sl], atom_seg, seg_coef,
                             Yin=None if Yin is None else Yin[:, sl])
        return out

    def __matmul__(self, X):
        return self.matmul(X)

    # -- test helpers ---------------------------------------------------------------
    def to_scipy_lower(self):
        """Lower triangle (incl. diagonal) as scipy CSR, FP64 (for tests only)."""
        import scipy.sparse as sp
        n = self.n_atoms
        rowptr = self.rowptr.cpu().numpy()
        cols = self.cols.cpu().numpy().astype(np.int64)
        ent = (self.ent64 if self.ent64 is not None else self.ent32.double()).cpu().numpy()
        diag = (self.diag64 if self.diag64 is not None else self.diag32.double()).cpu().numpy()
        rows = np.repeat(np.arange(n), np.diff(rowptr))
        w = ent[:, :3]
        blocks = -w[:, :, None] * w[:, None, :]
        D = np.zeros((n, 3, 3))
        D[:, 0, 0], D[:, 1, 1], D[:, 2, 2] = diag[:, 0], diag[:, 1], diag[:, 2]
        D[:, 0, 1] = D[:, 1, 0] = diag[:, 3]
        D[:, 0, 2] = D[:, 2, 0] = diag[:, 4]
        D[:, 1, 2] = D[:, 2, 1] = diag[:, 5]
        off = rows != cols
        bi = np.concatenate([rows[off], np.arange(n)])
        bj = np.concatenate([cols[off], np.arange(n)])
        bv = np.concatenate([blocks[off], D])
        p, q = np.meshgrid(np.arange(3), np.arange(3), indexing="ij")
        R = (3 * bi[:, None, None] + p[None]).ravel()
        C = (3 * bj[:, None, None] + q[None]).ravel()
        V = bv.ravel()
        keep = (C <= R) & (V != 0.0)
        A = sp.csr_matrix((V[keep], (R[keep], C[keep])), shape=self.shape)
        A.sum_duplicates()
        return A


def width_class(b):
    """Launch class of a b-column product: the kernel tile it mostly runs (128, 64,
    32 or 8 columns; narrower products are their own class)."""
    return 128 if b >= 128 else (64 if b >= 64 else (32 if b >= 32 else (8 if b >= 8 else b)))


def _band_aligned(m, vec):
    """Whether a (rows, b) block can go to the band kernel as it is: its data starts
    on 16 bytes and its leading dimension is a multiple of vec elements."""
    return m.data_ptr() % 16 == 0 and m.stride(1) == 1 and m.stride(0) % vec == 0


def _launches(b, prec):
    """SpMM kernel launches for b columns (tiles of 128/64/32/16/8/4/2/1 in FP32 per
    128-column panel, 32/16/8/4/2/1 in FP64 per 64-column panel)."""
    n = 0
    panel = 128 if prec == 32 else 64
    for c0 in range(0, b, panel):
        rem = min(panel, b - c0)
        for t in ((128, 64, 32, 16, 8, 4, 2, 1) if prec == 32 else (32, 16, 8, 4, 2, 1)):
            while rem >= t:
                rem -= t
                n += 1
    return n
