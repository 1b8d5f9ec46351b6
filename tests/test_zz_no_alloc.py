"""The allocation-free SpMM entry point (inch_spmm_noalloc) against the workspace
entry point (inch_spmm), called through the C ABI.

inch_spmm_noalloc exists for callers that cannot give the library device
scratch memory (a host that runs on another runtime's memory manager without a
device allocator of its own, or a thin FFI binding that only owns its inputs and
outputs): it keeps its deflation partial sums in a static device array instead.
Both entry points run the same kernels, so the outputs must agree to the FP64 /
FP32 tolerances of the other SpMM tests; two calls in a row check that the
shared static scratch carries nothing stale from one call into the next.

This file is collected last so that a run that stops at the first failure has
already run every other test; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {64: 1e-12, 32: 2e-6}


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


@pytest.fixture(scope="module")
def store():
    from inching_b200 import synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    X = synth.globule(2000, seed=31) / 10.0
    H = HessianStore(X, 8.0, plus_i=1.0)
    Q = rigid_body_basis(H.X)
    return H, Q


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("b", [1, 7, 40])
def test_noalloc_matches_workspace_entry(store, prec, b):
    from inching_b200 import _native
    H, Q = store
    L = _native.lib()
    n = H.shape[0]
    dt = torch.float64 if prec == 64 else torch.float32
    ent, diag = H.store(prec)
    g = torch.Generator(device="cuda")
    g.manual_seed(b)
    Xv = torch.randn((n, b), generator=g, dtype=torch.float64, device="cuda").to(dt).contiguous()
    Yin = torch.randn((n, b), generator=g, dtype=torch.float64, device="cuda").to(dt).contiguous()
    ep = _native.SpmmEpilogue(0.5, -0.25, -1.0, 0.0, 10.0, Q.shape[0], 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    ref = torch.empty_like(Xv)
    ws = torch.empty(L.inch_spmm_workspace_size(H.n_atoms, b, Q.shape[0]), dtype=torch.uint8, device="cuda")
    _native.check(L.inch_spmm(prec, H.n_atoms, _p(H.rowptr), _p(ent), _p(diag), _p(Xv), b, b, _p(ref), b,
                              _p(Yin), b, None, 0, _p(Q), ctypes.byref(ep), _p(ws), ws.numel(), stream))
    outs = []
    for _ in range(2):
        out = torch.full_like(Xv, float("nan"))
        _native.check(L.inch_spmm_noalloc(prec, H.n_atoms, _p(H.rowptr), _p(ent), _p(diag), _p(Xv), b, b,
                                          _p(out), b, _p(Yin), b, None, 0, _p(Q), ctypes.byref(ep), stream))
        outs.append(out)
    torch.cuda.synchronize()
    scale = float(ref.abs().max())
    for out in outs:
        assert torch.isfinite(out).all()
        assert float((out.double() - ref.double()).abs().max()) <= TOL[prec] * scale


def test_noalloc_rejects_sizes_beyond_its_scratch(store):
    from inching_b200 import _native
    H, Q = store
    L = _native.lib()
    n = H.shape[0]
    ent, diag = H.store(64)
    Xv = torch.zeros((n, 65), dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(Xv)
    ep = _native.SpmmEpilogue(1.0, 0.0, 0.0, 0.0, 0.0, 0, 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = L.inch_spmm_noalloc(64, H.n_atoms, _p(H.rowptr), _p(ent), _p(diag), _p(Xv), 65, 65, _p(Y), 65,
                             None, 0, None, 0, None, ctypes.byref(ep), stream)
    assert st == _native.INCH_LIMIT
    assert b"64 columns" in L.inch_last_error_string()
    Q9 = torch.zeros((9, n), dtype=torch.float64, device="cuda")
    ep9 = _native.SpmmEpilogue(1.0, 0.0, 0.0, 0.0, 1.0, 9, 0)
    st = L.inch_spmm_noalloc(64, H.n_atoms, _p(H.rowptr), _p(ent), _p(diag), _p(Xv), 65, 8, _p(Y), 65,
                             None, 0, None, 0, _p(Q9), ctypes.byref(ep9), stream)
    assert st == _native.INCH_LIMIT
