"""End-to-end normal modes: the driver flow of the reference as one call.

Mirrors the benchmark drivers (Command8A/commandBenchmark_InchingTRLMHD_Linux_Pdb_0064_A100.py:
212-407 and Notebook/Application/01_Inching_EigenproblemJDMHD.ipynb cell 4):
  1. coordinates in nm (PDB Angstrom / 10)
  2. reversed Cuthill-McKee order                     (X_KdCuthillMckeeOrder)
  3. Hessian H + PlusI*I of the reordered structure   (ReturnCupyHLowerTriangle)
  4. six rigid-body vectors for explicit deflation    (driver lines 314-372)
  5. eigensolver (TRLM / JDM / IRLM / CDM / block ChFSI)
  6. eigenvalues - PlusI, eigenvectors reshaped (k, N, 3) and put back in the
     caller's atom order                               (driver lines 396-407)
Everything from step 2 on runs on the GPU; `normal_modes` takes and returns host
arrays, `normal_modes_device` keeps inputs and results on the device.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import graph
from .deflation import rigid_body_basis
from .hessian import HessianStore

SOLVERS = ("chfsi", "trlm", "jdm", "irlm", "cdm")


def _solve(H, k, solver, precision, tol, Q, shift, seed, **kw):
    if solver == "chfsi":
        from .solvers.chfsi import chfsi
        return chfsi(H, k, tol=tol, Q=Q, precision=precision, seed=seed, return_info=True, **kw)
    if solver == "trlm":
        from .solvers.trlm import trlm
        return trlm(H, k=k, tol=tol, Q=Q, shift=shift, precision=precision, seed=seed, return_info=True, **kw)
    if solver == "jdm":
        from .solvers.jdm import jdm
        return jdm(H, k=k, tol=tol, Q=Q, shift=shift, precision=precision, seed=seed, return_info=True, **kw)
    if solver == "irlm":
        from .solvers.irlm import irlm
        return irlm(H, k=k, tol=tol, Q=Q, shift=shift, precision=precision, seed=seed, return_info=True, **kw)
    if solver == "cdm":
        from .solvers.cdm import cdm
        from .spectrum import estimate_spectrum_bound
        bound = kw.pop("spectrum_bound", None) or estimate_spectrum_bound(H, steps=300, seed=seed + 1)
        return cdm(H, k=k, tol=tol, Q=Q, precision=precision, spectrum_bound=bound, seed=seed, return_info=True,
                   **kw)
    raise AssertionError(f"ABORTED. unknown solver {solver!r}; use one of {SOLVERS}")


def normal_modes_device(X_nm: torch.Tensor, k: int, *, rc_gamma_A=8.0, plus_i=1.0, solver="chfsi",
                        precision="mixed", tol=1e-6, deflate_rigid=True, hotelling_shift=10.0, seed=0,
                        warm_start=None, pbc=None, **kw):
    """Lowest k non-rigid modes of the structure X_nm (CUDA (N,3) float64, nm).

    warm_start="coarse" (block solver only): initial block from the lowest modes
    of a bead model of the structure (inching_b200.warmstart); "galerkin": from the
    fine Hessian restricted to bead motions (P^T H P, the Rayleigh-Ritz-best bead
    block); "learned": the bead
    model's spring constants set by the trained network (inching_b200.learned;
    warm_model= a WarmStartMPNN, default the shipped weights), with its residual
    test and random-start fallback.

    tol: for "chfsi", the relative residual ||Hv - lambda v|| <= tol*||H||; for the
    reference solvers, their own absolute tolerance.  Returns (eigval (k,) with
    PlusI removed, eigvec (k, N, 3) in input atom order, info dict), on the GPU.

    pbc: periodic xy images (the reference's User_DictCharmmGuiPbc or
    (box_x, box_y) in nm); the deflated null space is then the three translations."""
    t0 = time.perf_counter()
    order, undo, (degree, _, _, levels) = graph.cuthill_mckee(X_nm, rc_gamma_A, return_graph=True, pbc=pbc)
    Xr = X_nm[order]
    precisions = ("f64", "f32") if precision == "mixed" else ("f64",)
    H = HessianStore(Xr, rc_gamma_A, plus_i=plus_i, precisions=precisions, pbc=pbc)
    if not deflate_rigid:
        Q = None
    elif pbc is not None:
        from .deflation import translation_basis
        Q = translation_basis(Xr.shape[0], device=Xr.device)
    else:
        Q = rigid_body_basis(Xr)
    if pbc is not None and warm_start is not None:
        raise AssertionError("ABORTED. the bead-model warm starts do not take periodic images")
    winfo = None
    if warm_start == "coarse":
        if solver != "chfsi":
            raise AssertionError("ABORTED. warm_start='coarse' is available for solver='chfsi'")
        from .warmstart import coarse_warm_start
        from .solvers.chfsi import default_guard
        # the starting block needs no tight coarse solve: tol 3e-3 kept the fine
        # iterations of 256 modes of 100k atoms at 4 and saved 10 ms against 1e-4;
        # only the k wanted bead modes converge, the guard columns stay Ritz vectors
        kw["X0"], winfo = coarse_warm_start(Xr, k + default_guard(k), tol=3e-3, seed=seed, return_info=True,
                                            wanted=k)
    elif warm_start == "galerkin":
        if solver != "chfsi":
            raise AssertionError("ABORTED. warm_start='galerkin' is available for solver='chfsi'")
        from .warmstart import galerkin_warm_start
        from .solvers.chfsi import default_guard
        kw["X0"], winfo = galerkin_warm_start(H, k + default_guard(k), seed=seed, return_info=True)
    elif warm_start == "learned":
        if solver != "chfsi":
            raise AssertionError("ABORTED. warm_start='learned' is available for solver='chfsi'")
        from .learned import WarmStartMPNN, learned_warm_start
        from .solvers.chfsi import default_guard
        kw["X0"], winfo = learned_warm_start(Xr, k + default_guard(k), kw.pop("warm_model", None) or
                                             WarmStartMPNN.load(device=X_nm.device), H.rowptr, H.cols,
                                             H=H, Q=Q, k=k, seed=seed, return_info=True)
    elif warm_start is not None:
        raise AssertionError(f"ABORTED. unknown warm_start {warm_start!r}")
    t1 = time.perf_counter()
    evals, evecs, info = _solve(H, k, solver, precision, tol, Q, hotelling_shift, seed, **kw)
    n_atoms = Xr.shape[0]
    modes = evecs.t().reshape(evecs.shape[1], n_atoms, 3)[:, undo, :]
    info = dict(info)
    info.update(dict(n_atoms=int(n_atoms), nnz_blocks=H.nnz_blocks, rcm_levels=levels,
                     mean_degree=float(degree.double().mean()), setup_s=t1 - t0, warm_start=winfo))
    return evals - plus_i, modes, info


def normal_modes(X, k: int, *, units="nm", **kw):
    """Host-facing call: X (N,3) numpy in nm (or Angstrom with units="A"); returns
    numpy eigenvalues (k,) (PlusI removed) and eigenvectors (k, N, 3) in the input
    atom order, plus an info dict."""
    Xh = np.asarray(X, dtype=np.float64)
    if units == "A":
        Xh = Xh / 10.0
    Xd = torch.from_numpy(np.ascontiguousarray(Xh)).pin_memory().to("cuda", non_blocking=True)
    evals, modes, info = normal_modes_device(Xd, k, **kw)
    ev = evals.cpu().numpy()
    # The (k, N, 3) float64 modes are read back into page-locked memory from torch's
    # caching host allocator: ~50 GB/s instead of ~2 GB/s into fresh pageable pages
    # (614 MB for 256 modes of 100k atoms: 12 ms instead of 0.3 s).  The returned
    # array keeps that block alive; it is reused only after the array is released.
    out = torch.empty(modes.shape, dtype=modes.dtype, pin_memory=True)
    out.copy_(modes, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return ev, out.numpy(), info
