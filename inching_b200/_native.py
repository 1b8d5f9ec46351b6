"""ctypes binding of libinching_b200.so (the C ABI declared in include/inching_b200.h).

There is no fallback: if the shared library is missing or CUDA is unavailable the
calls raise.  Device buffers are torch CUDA tensors passed by data pointer, on
torch's current stream; workspaces come from torch's caching allocator.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_double, c_int32, c_int64, c_size_t, c_void_p, c_char_p

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libinching_b200.so")

INCH_OK, INCH_INVALID_ARG, INCH_OOM, INCH_NOT_CONVERGED, INCH_TIMEOUT, INCH_CUDA_ERROR, INCH_LIMIT = range(7)
MAX_DEGREE = 1024


class InchError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"inching_b200 error {status}: {msg}")
        self.status = status


class CellGrid(Structure):
    _fields_ = [("origin", c_double * 3), ("cell", c_double), ("dims", c_int32 * 3),
                ("ncells", c_int64), ("n_atoms", c_int64)]


class SpmmEpilogue(Structure):
    _fields_ = [("alpha", c_double), ("gamma", c_double), ("beta", c_double), ("mu", c_double),
                ("hot_shift", c_double), ("r", c_int32), ("accumulate", c_int32)]


_lib = None

# Running count of kernels this binding has launched (each wrapper adds the
# number of kernels its entry point enqueues); read by measurement code.
launches = 0


def _count(n):
    global launches
    launches += int(n)

# name -> (restype, argtypes)
_SIGS = {
    "inch_last_error_string": (c_char_p, []),
    "inch_abi_version": (ctypes.c_int, []),
    "inch_cell_grid_plan": (ctypes.c_int, [c_void_p, c_int64, c_double, POINTER(CellGrid), c_void_p, c_size_t, c_void_p]),
    "inch_neighbors_workspace_size": (c_size_t, [POINTER(CellGrid)]),
    "inch_neighbors_count": (ctypes.c_int, [c_void_p, POINTER(CellGrid), c_double, c_void_p, c_void_p,
                                            POINTER(c_int64), c_void_p, c_size_t, c_void_p]),
    "inch_neighbors_fill": (ctypes.c_int, [c_void_p, POINTER(CellGrid), c_double, c_void_p, c_void_p,
                                           c_void_p, c_size_t, c_void_p]),
    "inch_neighbors_count_pbc_xy": (ctypes.c_int, [c_void_p, POINTER(CellGrid), c_double, c_double, c_double,
                                                   c_void_p, c_void_p, POINTER(c_int64), c_void_p, c_size_t,
                                                   c_void_p]),
    "inch_neighbors_fill_pbc_xy": (ctypes.c_int, [c_void_p, POINTER(CellGrid), c_double, c_double, c_double,
                                                  c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "inch_cheb_filter": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32,
                                        c_int32, POINTER(c_double), c_double, c_double, c_void_p, c_int64, c_void_p,
                                        c_void_p, c_int64, c_void_p]),
    "inch_cheb_filter_scaled": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                               c_int32, c_int32, c_double, c_double, c_double, c_void_p, c_int64,
                                               c_void_p, c_int64, c_void_p]),
    "inch_block_orth_workspace_size": (c_size_t, [c_int32, c_int64]),
    "inch_block_orth": (ctypes.c_int, [c_int64, c_int32, c_void_p, c_int64, c_void_p, c_int64, c_int64, c_void_p,
                                       c_int64, c_int64, c_int32, c_void_p, c_size_t, c_void_p]),
    "inch_rr_workspace_size": (c_size_t, []),
    "inch_rr_project": (ctypes.c_int, [c_int64, c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p,
                                       c_size_t, c_void_p]),
    "inch_rr_rotate": (ctypes.c_int, [c_int64, c_int32, c_int32, c_void_p, c_int64, c_void_p, c_void_p, c_int64,
                                      c_void_p, c_size_t, c_void_p]),
    "inch_residual_workspace_size": (c_size_t, [c_int32]),
    "inch_residual_fp64": (ctypes.c_int, [c_int64, c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p,
                                          c_void_p, c_size_t, c_void_p]),
    "inch_eigh_batched_small": (ctypes.c_int, [c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_int32, c_double,
                                               c_void_p, c_void_p]),
    "inch_hessian_assemble_pbc_xy": (ctypes.c_int, [c_void_p, c_int64, c_double, c_double, c_void_p, c_void_p,
                                                    c_void_p, c_double, c_double, c_void_p, c_void_p, c_void_p,
                                                    c_void_p, c_void_p]),
    "inch_rcm_workspace_size": (c_size_t, [c_int64]),
    "inch_rcm": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p,
                                POINTER(c_int32), c_void_p, c_size_t, c_void_p]),
    "inch_band_slices_workspace_size": (c_size_t, [c_int64, c_int64]),
    "inch_band_slices": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_int64, c_int32,
                                        c_void_p, c_void_p, c_void_p, POINTER(c_int64), c_void_p, c_size_t,
                                        c_void_p]),
    "inch_hessian_assemble": (ctypes.c_int, [c_void_p, c_int64, c_double, c_double, c_void_p, c_void_p,
                                             c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "inch_spmm_workspace_size": (c_size_t, [c_int64, c_int32, c_int32]),
    "inch_spmm_tune": (ctypes.c_int, [c_int32, c_int32]),
    "inch_spmm_traversal": (ctypes.c_int, [c_int32]),
    "inch_spmm_seg": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32,
                                     c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_void_p]),
    "inch_spmm_seg_ws": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32,
                                        c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_size_t,
                                        c_void_p]),
    "inch_spmm": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32,
                                 c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                 POINTER(SpmmEpilogue), c_void_p, c_size_t, c_void_p]),
    "inch_tile_store_workspace_size": (c_size_t, [c_int64]),
    "inch_tile_store_count": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, POINTER(c_int64),
                                             POINTER(c_int64), c_void_p, c_size_t, c_void_p]),
    "inch_tile_store_fill": (ctypes.c_int, [c_void_p, c_int64, c_double, c_void_p, c_void_p, c_void_p, c_void_p,
                                            c_void_p, c_void_p, c_void_p, c_void_p]),
    "inch_spmm_tiles_workspace_size": (c_size_t, []),
    "inch_spmm_tiles": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_int64, c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                       c_int64, c_void_p, POINTER(SpmmEpilogue), c_void_p, c_size_t, c_void_p]),
    "inch_spmm_tiles_seg": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_void_p, c_int64, c_int32, c_void_p, c_int64, c_void_p, c_int64,
                                           c_void_p, c_void_p, c_void_p]),
    "inch_group_store_workspace_size": (c_size_t, [c_int64, c_int32]),
    "inch_group_store_count": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_int32, c_void_p, POINTER(c_int64),
                                              c_void_p, c_size_t, c_void_p]),
    "inch_group_store_fill": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p]),
    "inch_spmm_group_tune": (ctypes.c_int, [c_int32]),
    "inch_spmm_groups": (ctypes.c_int, [c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32,
                                        c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                        POINTER(SpmmEpilogue), c_void_p, c_size_t, c_void_p]),
    "inch_spmm_groups_seg": (ctypes.c_int, [c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                            c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p,
                                            c_void_p, c_size_t, c_void_p]),
    "inch_spmm_band_tune": (ctypes.c_int, [c_int32]),
    "inch_spmm_band_status": (ctypes.c_int, [POINTER(c_int32)]),
    "inch_hessian_assemble_weighted": (ctypes.c_int, [c_void_p, c_int64, c_double, c_double, c_void_p, c_void_p,
                                                      c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "inch_mp_edge_concat": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_int32, c_void_p,
                                           c_void_p]),
    "inch_mp_edge_concat_bwd": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_int32, c_int32, c_void_p, c_void_p]),
    "inch_mp_segment_sum": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p]),
    "inch_mp_segment_sum_bwd": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p]),
    "inch_mp_bias_relu": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_int32, c_void_p]),
    "inch_mp_relu_bwd": (ctypes.c_int, [c_void_p, c_void_p, c_int64, c_void_p]),
    "inch_mp_edge_pair": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_int32,
                                         c_void_p, c_void_p]),
    "inch_mp_edge_pair_bwd": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_int32, c_void_p,
                                             c_void_p]),
    "inch_mp_softplus": (ctypes.c_int, [c_void_p, c_int64, ctypes.c_float, c_void_p, c_void_p, c_void_p, c_void_p]),
    "inch_mp_hf_grad": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                       c_int64, c_void_p, c_void_p]),
    "inch_mp_adam": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_float, c_int32, c_void_p]),
    "inch_mp_gemm_workspace_size": (c_size_t, [c_int32, c_int32, c_int32]),
    "inch_mp_gemm": (ctypes.c_int, [c_int32, c_int32, c_int32, c_void_p, c_int64, c_int64, c_void_p, c_int64, c_int64,
                                    c_void_p, c_int64, ctypes.c_float, c_void_p, c_size_t, c_void_p]),
    "inch_spmm_noalloc": (ctypes.c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                         c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64,
                                         c_void_p, POINTER(SpmmEpilogue), c_void_p]),
}


def exported_symbols():
    """Names of the C-ABI entry points this binding declares."""
    return sorted(_SIGS)


def lib():
    """Load the shared library once; raise if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m inching_b200.build` "
                          "(the CUDA path has no fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int):
    if status == INCH_OK:
        return
    msg = lib().inch_last_error_string().decode(errors="replace")
    if status == INCH_INVALID_ARG:
        raise AssertionError(msg if msg.startswith("ABORTED") else "ABORTED. " + msg)
    raise InchError(status, msg)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ws(nbytes, device):
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def _require_cuda(t, name, dtype=None):
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise AssertionError(f"ABORTED. {name} must be a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise AssertionError(f"ABORTED. {name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise AssertionError(f"ABORTED. {name} must be contiguous")


# ---------------------------------------------------------------------------
# Neighbours, Cuthill-McKee, band slices
# ---------------------------------------------------------------------------
def neighbor_lists(X: torch.Tensor, rc_nm: float, box_xy=None):
    """(degree int32 (N,), rowptr int64 (N+1,), cols int32 (nnz,)) on X's device;
    with box_xy = (box_x, box_y) in nm, periodic xy images too, and a fourth
    tensor: the image code (int8, nnz) of every entry."""
    _require_cuda(X, "X", torch.float64)
    L = lib()
    n = X.shape[0]
    dev = X.device
    grid = CellGrid()
    w0 = _ws(256, dev)
    check(L.inch_cell_grid_plan(_ptr(X), n, rc_nm, ctypes.byref(grid), _ptr(w0), w0.numel(), _stream()))
    ws = _ws(L.inch_neighbors_workspace_size(ctypes.byref(grid)), dev)
    degree = torch.empty(n, dtype=torch.int32, device=dev)
    rowptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
    nnz = c_int64(0)
    if box_xy is None:
        check(L.inch_neighbors_count(_ptr(X), ctypes.byref(grid), rc_nm, _ptr(degree), _ptr(rowptr),
                                     ctypes.byref(nnz), _ptr(ws), ws.numel(), _stream()))
    else:
        bx, by = float(box_xy[0]), float(box_xy[1])
        check(L.inch_neighbors_count_pbc_xy(_ptr(X), ctypes.byref(grid), rc_nm, bx, by, _ptr(degree), _ptr(rowptr),
                                            ctypes.byref(nnz), _ptr(ws), ws.numel(), _stream()))
    cols = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)[:nnz.value]
    _count(8)   # bbox, assign, scan, scatter, count, set0, scan, fill
    if box_xy is None:
        check(L.inch_neighbors_fill(_ptr(X), ctypes.byref(grid), rc_nm, _ptr(rowptr), _ptr(cols),
                                    _ptr(ws), ws.numel(), _stream()))
        return degree, rowptr, cols
    image = torch.empty(max(nnz.value, 1), dtype=torch.int8, device=dev)[:nnz.value]
    check(L.inch_neighbors_fill_pbc_xy(_ptr(X), ctypes.byref(grid), rc_nm, bx, by, _ptr(rowptr), _ptr(cols),
                                       _ptr(image), _ptr(ws), ws.numel(), _stream()))
    return degree, rowptr, cols, image


def cuthill_mckee(rowptr, cols, degree, seed_order):
    """Reversed Cuthill-McKee order and its inverse (int64 device tensors), levels."""
    for t, nm, dt in ((rowptr, "rowptr", torch.int64), (cols, "cols", torch.int32),
                      (degree, "degree", torch.int32), (seed_order, "seed_order", torch.int64)):
        _require_cuda(t, nm, dt)
    L = lib()
    n = degree.shape[0]
    dev = degree.device
    ws = _ws(L.inch_rcm_workspace_size(n), dev)
    order = torch.empty(n, dtype=torch.int64, device=dev)
    undo = torch.empty(n, dtype=torch.int64, device=dev)
    levels = c_int32(0)
    check(L.inch_rcm(_ptr(rowptr), _ptr(cols), _ptr(degree), _ptr(seed_order), n, _ptr(order), _ptr(undo),
                     ctypes.byref(levels), _ptr(ws), ws.numel(), _stream()))
    _count(5 + 5 * levels.value)
    return order, undo, levels.value


def band_slices(rowptr, cols, n_atoms, heads, gap=100, max_slices=256):
    """Per-batch (counts int32, starts int64 (nb, max_slices), ends, total neighbours)."""
    _require_cuda(rowptr, "rowptr", torch.int64)
    _require_cuda(cols, "cols", torch.int32)
    _require_cuda(heads, "heads", torch.int64)
    L = lib()
    nb = heads.shape[0] - 1
    dev = rowptr.device
    nnz = int(rowptr[n_atoms].item())
    ws = _ws(L.inch_band_slices_workspace_size(nb, nnz), dev)
    starts = torch.empty((nb, max_slices), dtype=torch.int64, device=dev)
    ends = torch.empty((nb, max_slices), dtype=torch.int64, device=dev)
    counts = torch.empty(nb, dtype=torch.int32, device=dev)
    total = c_int64(0)
    check(L.inch_band_slices(_ptr(rowptr), _ptr(cols), n_atoms, _ptr(heads), nb, gap, max_slices, _ptr(starts),
                             _ptr(ends), _ptr(counts), ctypes.byref(total), _ptr(ws), ws.numel(), _stream()))
    return counts, starts, ends, total.value


# ---------------------------------------------------------------------------
# Hessian store and operator
# ---------------------------------------------------------------------------
def hessian_assemble(X, rowptr, cols, rc_nm, plus_i, want64=True, want32=True, pair_weight=None, image=None,
                     box_xy=None):
    _require_cuda(X, "X", torch.float64)
    _require_cuda(rowptr, "rowptr", torch.int64)
    _require_cuda(cols, "cols", torch.int32)
    n = X.shape[0]
    nnz = cols.shape[0]
    dev = X.device
    ent64 = torch.empty((nnz, 4), dtype=torch.float64, device=dev) if want64 else None
    diag64 = torch.empty((n, 8), dtype=torch.float64, device=dev) if want64 else None
    ent32 = torch.empty((nnz, 4), dtype=torch.float32, device=dev) if want32 else None
    diag32 = torch.empty((n, 8), dtype=torch.float32, device=dev) if want32 else None
    if image is not None:
        assert pair_weight is None, "ABORTED. periodic images and pair weights are not combined"
        _require_cuda(image, "image", torch.int8)
        if image.numel() != nnz:
            raise AssertionError(f"ABORTED. image holds {image.numel()} codes for {nnz} adjacency entries")
        check(lib().inch_hessian_assemble_pbc_xy(_ptr(X), n, rc_nm, plus_i, _ptr(rowptr), _ptr(cols), _ptr(image),
                                                 float(box_xy[0]), float(box_xy[1]), _ptr(ent64), _ptr(diag64),
                                                 _ptr(ent32), _ptr(diag32), _stream()))
    elif pair_weight is None:
        check(lib().inch_hessian_assemble(_ptr(X), n, rc_nm, plus_i, _ptr(rowptr), _ptr(cols), _ptr(ent64),
                                          _ptr(diag64), _ptr(ent32), _ptr(diag32), _stream()))
    else:
        _require_cuda(pair_weight, "pair_weight", torch.float64)
        if pair_weight.numel() != nnz:
            raise AssertionError(f"ABORTED. pair_weight holds {pair_weight.numel()} springs for {nnz} adjacency "
                                 "entries")
        if bool((pair_weight < 0).any()):
            raise AssertionError("ABORTED. pair_weight must be non-negative (each block is -gamma u u^T)")
        check(lib().inch_hessian_assemble_weighted(_ptr(X), n, rc_nm, plus_i, _ptr(rowptr), _ptr(cols),
                                                   _ptr(pair_weight), _ptr(ent64), _ptr(diag64), _ptr(ent32),
                                                   _ptr(diag32), _stream()))
    _count(1)
    return ent64, diag64, ent32, diag32


_ws_cache = {}


def spmm_seg(prec, n_atoms, rowptr, ent, diag, X, Y, atom_seg, seg_coef, Yin=None):
    """Y = alpha_s (H X) + gamma_s X + beta_s Yin with (alpha, gamma, beta) per segment s
    of atom i (atom_seg int32 (N,), seg_coef float64 (S, 3)).  X, Y: (3N, b), b <= 128
    (FP32) / 64 (FP64); runs with the device's cached workspace (row counter)."""
    L = lib()
    b = 1 if X.dim() == 1 else X.shape[1]
    ldx = 1 if X.dim() == 1 else X.stride(0)
    ldy = 1 if Y.dim() == 1 else Y.stride(0)
    ldyin = 0 if Yin is None else (1 if Yin.dim() == 1 else Yin.stride(0))
    dev = X.device
    ws = _ws_cache.get((dev.index, False))
    if ws is None:
        ws = _ws(L.inch_spmm_workspace_size(n_atoms, b, 0), dev)
        _ws_cache[(dev.index, False)] = ws
    check(L.inch_spmm_seg_ws(prec, n_atoms, _ptr(rowptr), _ptr(ent), _ptr(diag), _ptr(X), ldx, b, _ptr(Y), ldy,
                             _ptr(Yin), ldyin, _ptr(atom_seg), _ptr(seg_coef), _ptr(ws), ws.numel(), _stream()))
    tiles = 0
    rem = b
    for t in ((128, 64, 32, 16, 8, 4, 2, 1) if prec == 32 else (32, 16, 8, 4, 2, 1)):
        while rem >= t:
            rem -= t
            tiles += 1
    _count(tiles)
    return Y


_spmm_setting = [None]


def spmm_tune(threads_per_block=256, blocks_per_sm=5, traversal=None):
    """Set the wide-block SpMM launch shape (and, if given, the row traversal: 0
    fixed stride, 1 per-warp chunks, 2 per-block chunks) for this process
    (autotuner hook)."""
    setting = (threads_per_block, blocks_per_sm, traversal)
    if _spmm_setting[0] == setting:
        return
    check(lib().inch_spmm_tune(threads_per_block, blocks_per_sm))
    if traversal is not None:
        check(lib().inch_spmm_traversal(traversal))
    _spmm_setting[0] = setting


def spmm(prec, n_atoms, rowptr, ent, diag, X, Y, *, alpha=1.0, gamma=0.0, beta=0.0, Yin=None,
         acc=None, mu=0.0, Q=None, hot_shift=0.0):
    """Y = alpha*(H X) + gamma*X + beta*Yin + hot_shift*Q^T(Q X); acc += mu*Y if acc given.

    X, Y, Yin, acc: (3N,) or (3N, b) tensors whose last dimension is contiguous."""
    L = lib()
    b = 1 if X.dim() == 1 else X.shape[1]
    ldx = 1 if X.dim() == 1 else X.stride(0)
    ldy = 1 if Y.dim() == 1 else Y.stride(0)
    ldyin = 0 if Yin is None else (1 if Yin.dim() == 1 else Yin.stride(0))
    ldacc = 0 if acc is None else (1 if acc.dim() == 1 else acc.stride(0))
    r = 0 if Q is None else Q.shape[0]
    ep = SpmmEpilogue(alpha, gamma, beta, mu, hot_shift, r, 1 if acc is not None else 0)
    dev = X.device
    key = (dev.index, r > 0)
    ws = _ws_cache.get(key)
    if ws is None:
        ws = _ws(L.inch_spmm_workspace_size(n_atoms, b, r), dev)
        _ws_cache[key] = ws
    check(L.inch_spmm(prec, n_atoms, _ptr(rowptr), _ptr(ent), _ptr(diag), _ptr(X), ldx, b, _ptr(Y), ldy,
                      _ptr(Yin), ldyin, _ptr(acc), ldacc, _ptr(Q), ctypes.byref(ep), _ptr(ws), ws.numel(),
                      _stream()))
    tiles = 0
    rem = b
    for t in ((128, 64, 32, 16, 8, 4, 2, 1) if prec == 32 else (32, 16, 8, 4, 2, 1)):
        while rem >= t:
            rem -= t
            tiles += 1
    _count(tiles * (3 if r > 0 else 1))
    return Y


# ---------------------------------------------------------------------------
# Row-tile store (wide multivectors)
# ---------------------------------------------------------------------------
def tile_store(X, rowptr, cols, rc_nm, want64=True, want32=True):
    """(tile_uptr, tile_pptr, urec, pw64, pw32, n_union, n_pairs) for 8-row tiles."""
    L = lib()
    n = X.shape[0]
    dev = X.device
    nt = (n + 7) // 8
    uptr = torch.empty(nt + 1, dtype=torch.int64, device=dev)
    pptr = torch.empty(nt + 1, dtype=torch.int64, device=dev)
    ws = _ws(L.inch_tile_store_workspace_size(n), dev)
    nu, npairs = c_int64(0), c_int64(0)
    check(L.inch_tile_store_count(_ptr(rowptr), _ptr(cols), n, _ptr(uptr), _ptr(pptr), ctypes.byref(nu),
                                  ctypes.byref(npairs), _ptr(ws), ws.numel(), _stream()))
    urec = torch.empty(max(nu.value, 1), dtype=torch.int32, device=dev)
    pw64 = torch.empty((max(npairs.value, 1), 4), dtype=torch.float64, device=dev) if want64 else None
    pw32 = torch.empty((max(npairs.value, 1), 4), dtype=torch.float32, device=dev) if want32 else None
    check(L.inch_tile_store_fill(_ptr(X), n, rc_nm, _ptr(rowptr), _ptr(cols), _ptr(uptr), _ptr(pptr), _ptr(urec),
                                 _ptr(pw64), _ptr(pw32), _stream()))
    _count(4)
    return uptr, pptr, urec, pw64, pw32, nu.value, npairs.value


_tws = {}


def spmm_tiles(prec, n_atoms, uptr, pptr, urec, pw, diag, X, Y, *, alpha=1.0, gamma=0.0, beta=0.0, Yin=None,
               acc=None, mu=0.0, Q=None, hot_shift=0.0):
    """Same contract as spmm(), on the row-tile store."""
    L = lib()
    b = 1 if X.dim() == 1 else X.shape[1]
    ldx = 1 if X.dim() == 1 else X.stride(0)
    ldy = 1 if Y.dim() == 1 else Y.stride(0)
    ldyin = 0 if Yin is None else (1 if Yin.dim() == 1 else Yin.stride(0))
    ldacc = 0 if acc is None else (1 if acc.dim() == 1 else acc.stride(0))
    r = 0 if Q is None else Q.shape[0]
    ep = SpmmEpilogue(alpha, gamma, beta, mu, hot_shift, r, 1 if acc is not None else 0)
    dev = X.device
    ws = _tws.get(dev.index)
    if ws is None:
        ws = _ws(L.inch_spmm_tiles_workspace_size(), dev)
        _tws[dev.index] = ws
    check(L.inch_spmm_tiles(prec, n_atoms, _ptr(uptr), _ptr(pptr), _ptr(urec), _ptr(pw), _ptr(diag), _ptr(X), ldx,
                            b, _ptr(Y), ldy, _ptr(Yin), ldyin, _ptr(acc), ldacc, _ptr(Q), ctypes.byref(ep),
                            _ptr(ws), ws.numel(), _stream()))
    _count(band_panels(prec, b) * (3 if r > 0 else 1))
    return Y


_band_widest32 = 128


def band_panels(prec, b):
    """Kernel launches of one band-tile product of b columns: panels of 128 (FP32,
    when selected), 64 and 32 columns, the last one partial."""
    n = 0
    rem = b
    for w in (((_band_widest32, 64) if _band_widest32 == 128 else (64,)) if prec == 32 else (64,)):
        while rem >= w:
            rem -= w
            n += 1
    return n + (rem + 31) // 32


def spmm_band_tune(widest_fp32_panel=128):
    """Widest FP32 panel of the band-tile product for this process: 128 or 64."""
    global _band_widest32
    check(lib().inch_spmm_band_tune(widest_fp32_panel))
    _band_widest32 = int(widest_fp32_panel)


def spmm_band_status():
    """0, or 1 if a band-tile launch since the last call stopped at a bounded wait
    (synchronises; reading clears it)."""
    v = c_int32(0)
    check(lib().inch_spmm_band_status(ctypes.byref(v)))
    return int(v.value)


def spmm_tiles_seg(prec, n_atoms, uptr, pptr, urec, pw, diag, X, Y, atom_seg, seg_coef, Yin=None):
    """spmm_seg() on the row-tile store (any number of columns)."""
    L = lib()
    b = 1 if X.dim() == 1 else X.shape[1]
    ldx = 1 if X.dim() == 1 else X.stride(0)
    ldy = 1 if Y.dim() == 1 else Y.stride(0)
    ldyin = 0 if Yin is None else (1 if Yin.dim() == 1 else Yin.stride(0))
    check(L.inch_spmm_tiles_seg(prec, n_atoms, _ptr(uptr), _ptr(pptr), _ptr(urec), _ptr(pw), _ptr(diag), _ptr(X),
                                ldx, b, _ptr(Y), ldy, _ptr(Yin), ldyin, _ptr(atom_seg), _ptr(seg_coef), _stream()))
    _count(band_panels(prec, b))
    return Y


# ---------------------------------------------------------------------------
# Row-group store (FP32; R consecutive rows merged over their neighbour lists)
# ---------------------------------------------------------------------------
def group_store(rowptr, ent32, n_atoms, rows_per_group=2):
    """(group_ptr int64 (G+1,), group_ent float32 (U*R, 4), n_union) built from the
    FP32 pair entries: R = 2 or 4 consecutive rows per group, each group's unions
    padded to a multiple of 16."""
    L = lib()
    _require_cuda(ent32, "ent32", torch.float32)
    R = int(rows_per_group)
    if R not in (2, 4):
        raise AssertionError("ABORTED. rows_per_group must be 2 or 4")
    dev = ent32.device
    ng = (n_atoms + R - 1) // R
    gptr = torch.empty(ng + 1, dtype=torch.int64, device=dev)
    ws = _ws(L.inch_group_store_workspace_size(n_atoms, R), dev)
    nu = c_int64(0)
    check(L.inch_group_store_count(_ptr(rowptr), _ptr(ent32), n_atoms, R, _ptr(gptr), ctypes.byref(nu), _ptr(ws),
                                   ws.numel(), _stream()))
    gent = torch.empty((max(nu.value, 1) * R, 4), dtype=torch.float32, device=dev)
    check(L.inch_group_store_fill(_ptr(rowptr), _ptr(ent32), n_atoms, R, _ptr(gptr), _ptr(gent), _stream()))
    _count(4)
    return gptr, gent, nu.value


def group_tiles(b, aligned4=True, aligned2=True):
    """Kernel tiles of one row-group product of b columns (128 / 64 / 32, the last
    one partial)."""
    n, c0 = 0, 0
    while c0 < b:
        rem = b - c0
        if rem >= 128 and aligned4:
            c0 += 128
        elif rem >= 64 and aligned2:
            c0 += 64
        else:
            c0 += min(rem, 32)
        n += 1
    return n


def _aligned(m, k):
    if m is None:
        return True
    ld = 1 if m.dim() == 1 else m.stride(0)
    return ld % k == 0 and m.data_ptr() % (4 * k) == 0


def spmm_group_tune(unroll=0):
    """Unions in flight per warp of the row-group product (0: the default, 16 on
    128-column tiles and 8 on narrower ones; or 2, 4, 8, 16) for this process
    (autotuner hook)."""
    check(lib().inch_spmm_group_tune(int(unroll)))


def spmm_groups(n_atoms, rows_per_group, gptr, gent, diag, X, Y, *, alpha=1.0, gamma=0.0, beta=0.0, Yin=None,
                acc=None, mu=0.0, Q=None, hot_shift=0.0):
    """Same contract as spmm() in FP32, on the row-group store (any number of columns)."""
    L = lib()
    b = 1 if X.dim() == 1 else X.shape[1]
    ldx = 1 if X.dim() == 1 else X.stride(0)
    ldy = 1 if Y.dim() == 1 else Y.stride(0)
    ldyin = 0 if Yin is None else (1 if Yin.dim() == 1 else Yin.stride(0))
    ldacc = 0 if acc is None else (1 if acc.dim() == 1 else acc.stride(0))
    r = 0 if Q is None else Q.shape[0]
    ep = SpmmEpilogue(alpha, gamma, beta, mu, hot_shift, r, 1 if acc is not None else 0)
    dev = X.device
    key = (dev.index, r > 0)
    ws = _ws_cache.get(key)
    if ws is None:
        ws = _ws(L.inch_spmm_workspace_size(n_atoms, b, r), dev)
        _ws_cache[key] = ws
    check(L.inch_spmm_groups(n_atoms, rows_per_group, _ptr(gptr), _ptr(gent), _ptr(diag), _ptr(X), ldx, b, _ptr(Y),
                             ldy, _ptr(Yin), ldyin, _ptr(acc), ldacc, _ptr(Q), ctypes.byref(ep), _ptr(ws),
                             ws.numel(), _stream()))
    blocks = [X, Y] + ([Yin] if beta != 0.0 else []) + ([acc] if acc is not None else [])
    nt = group_tiles(b, all(_aligned(m, 4) for m in blocks), all(_aligned(m, 2) for m in blocks))
    _count(nt * (3 if r > 0 else 1))
    return Y


def spmm_groups_seg(n_atoms, rows_per_group, gptr, gent, diag, X, Y, atom_seg, seg_coef, Yin=None):
    """spmm_seg() on the row-group store (FP32, any number of columns)."""
    L = lib()
    b = 1 if X.dim() == 1 else X.shape[1]
    ldx = 1 if X.dim() == 1 else X.stride(0)
    ldy = 1 if Y.dim() == 1 else Y.stride(0)
    ldyin = 0 if Yin is None else (1 if Yin.dim() == 1 else Yin.stride(0))
    dev = X.device
    ws = _ws_cache.get((dev.index, False))
    if ws is None:
        ws = _ws(L.inch_spmm_workspace_size(n_atoms, b, 0), dev)
        _ws_cache[(dev.index, False)] = ws
    check(L.inch_spmm_groups_seg(n_atoms, rows_per_group, _ptr(gptr), _ptr(gent), _ptr(diag), _ptr(X), ldx, b,
                                 _ptr(Y), ldy, _ptr(Yin), ldyin, _ptr(atom_seg), _ptr(seg_coef), _ptr(ws),
                                 ws.numel(), _stream()))
    blocks = [X, Y] + ([Yin] if Yin is not None else [])
    _count(group_tiles(b, all(_aligned(m, 4) for m in blocks), all(_aligned(m, 2) for m in blocks)))
    return Y


# ---------------------------------------------------------------------------
# Message-passing network kernels (learned warm start)
# ---------------------------------------------------------------------------
_gemm_ws = {}


def mp_gemm(A, B, C, beta=0.0):
    """C = A B + beta C (FP32) with the package's dense-layer kernel; A, B may be any
    strided 2-D views (transposes included), C row-major with unit column stride."""
    for t, nm in ((A, "A"), (B, "B"), (C, "C")):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.dim() == 2):
            raise AssertionError(f"ABORTED. {nm} must be a 2-D float32 CUDA tensor")
    M, K = A.shape
    K2, N = B.shape
    if K2 != K or tuple(C.shape) != (M, N) or C.stride(1) != 1:
        raise AssertionError("ABORTED. mp_gemm: shapes or output layout do not match")
    L = lib()
    need = L.inch_mp_gemm_workspace_size(M, N, K)
    dev = C.device.index
    ws = _gemm_ws.get(dev)
    if ws is None or ws.numel() < need:
        ws = _ws(need, C.device)
        _gemm_ws[dev] = ws
    check(L.inch_mp_gemm(M, N, K, _ptr(A), A.stride(0), A.stride(1), _ptr(B), B.stride(0), B.stride(1), _ptr(C),
                         C.stride(0), float(beta), _ptr(ws), ws.numel(), _stream()))
    _count(1 if need <= 256 else 2)
    return C


def mp(name, *args):
    """Call inch_mp_<name>(*args, stream): tensors become device pointers."""
    conv = [(_ptr(a) if isinstance(a, torch.Tensor) else a) for a in args]
    check(getattr(lib(), "inch_mp_" + name)(*conv, _stream()))
    _count(1)


# ---------------------------------------------------------------------------
# Solver building blocks (C-ABI forms; the Python solvers use torch for the same
# dense steps, these serve non-Python hosts and are checked against them)
# ---------------------------------------------------------------------------
def _ld(t):
    return 1 if t.dim() == 1 else t.stride(0)


def cheb_filter(prec, n_atoms, rowptr, ent, diag, X, mu, cc, dd):
    """Y = sum_k mu[k] T_k((H - cc)/dd) X through inch_cheb_filter."""
    b = X.shape[1]
    Y = torch.empty_like(X)
    W1 = torch.empty_like(X)
    W2 = torch.empty_like(X)
    mu_h = (c_double * len(mu))(*[float(m) for m in mu])
    check(lib().inch_cheb_filter(prec, n_atoms, _ptr(rowptr), _ptr(ent), _ptr(diag), _ptr(X), _ld(X), b,
                                 len(mu) - 1, mu_h, cc, dd, _ptr(Y), _ld(Y), _ptr(W1), _ptr(W2), _ld(W1), _stream()))
    _count(len(mu) + 1)
    return Y


def cheb_filter_scaled(prec, n_atoms, rowptr, ent, diag, X, degree, a, b_up, a0):
    b = X.shape[1]
    Y = torch.empty_like(X)
    W = torch.empty_like(X)
    check(lib().inch_cheb_filter_scaled(prec, n_atoms, _ptr(rowptr), _ptr(ent), _ptr(diag), _ptr(X), _ld(X), b,
                                        degree, a, b_up, a0, _ptr(Y), _ld(Y), _ptr(W), _ld(W), _stream()))
    _count(degree + 1)
    return Y


def block_orth(Y, B1=None, B2=None, passes=2):
    """In place: Y <- orthonormal basis of (I - B B^T) Y (FP64, row bases B1, B2)."""
    _require_cuda(Y, "Y", torch.float64)
    n, b = Y.shape
    r1 = 0 if B1 is None else B1.shape[0]
    r2 = 0 if B2 is None else B2.shape[0]
    L = lib()
    ws = _ws(L.inch_block_orth_workspace_size(b, max(r1, r2)), Y.device)
    check(L.inch_block_orth(n, b, _ptr(Y), _ld(Y), _ptr(B1), r1, 0 if B1 is None else B1.stride(0), _ptr(B2), r2,
                            0 if B2 is None else B2.stride(0), passes, _ptr(ws), ws.numel(), _stream()))
    return Y


def rr_project(Y, HY):
    n, b = Y.shape
    G = torch.empty((b, b), dtype=torch.float64, device=Y.device)
    L = lib()
    ws = _ws(L.inch_rr_workspace_size(), Y.device)
    check(L.inch_rr_project(n, b, _ptr(Y), _ld(Y), _ptr(HY), _ld(HY), _ptr(G), _ptr(ws), ws.numel(), _stream()))
    return G          # column-major storage of a symmetric matrix: same values either way


def rr_rotate(Y, W, m):
    """Z = Y W[:, :m] for W with eigenvectors in columns (torch/numpy convention)."""
    n, b = Y.shape
    Wc = W.t().contiguous()          # column-major W
    Z = torch.empty((n, m), dtype=torch.float64, device=Y.device)
    L = lib()
    ws = _ws(L.inch_rr_workspace_size(), Y.device)
    check(L.inch_rr_rotate(n, b, m, _ptr(Y), _ld(Y), _ptr(Wc), _ptr(Z), _ld(Z), _ptr(ws), ws.numel(), _stream()))
    return Z


def residual_fp64(HY, Y, theta):
    n, b = Y.shape
    res = torch.empty(b, dtype=torch.float64, device=Y.device)
    L = lib()
    ws = _ws(L.inch_residual_workspace_size(b), Y.device)
    check(L.inch_residual_fp64(n, b, _ptr(HY), _ld(HY), _ptr(Y), _ld(Y), _ptr(theta.contiguous()), _ptr(res),
                               _ptr(ws), ws.numel(), _stream()))
    _count(2)
    return res


def eigh_batched_small(G, max_sweeps=30, tol=1e-13, return_sweeps=False):
    """Eigenpairs of a (S, p, p) stack of symmetric FP64 device matrices, p <= 64:
    (W (S, p) ascending, V (S, p, p) eigenvectors in columns), one CTA per matrix."""
    _require_cuda(G, "G", torch.float64)
    S, p, _ = G.shape
    W = torch.empty((S, p), dtype=torch.float64, device=G.device)
    V = torch.empty((S, p, p), dtype=torch.float64, device=G.device)
    sw = torch.empty(S, dtype=torch.int32, device=G.device) if return_sweeps else None
    check(lib().inch_eigh_batched_small(_ptr(G), S, p, _ptr(W), _ptr(V), max_sweeps, tol, _ptr(sw), _stream()))
    _count(1)
    return (W, V, sw) if return_sweeps else (W, V)
