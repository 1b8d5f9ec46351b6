"""Many modes at constant memory: the interval-marching filtered-TRLM driver
(the reference's many-mode application, Notebook/Application/
04_Inching_EigenproblemManyCTRLM.ipynb, driver cell lines 182-433), on this
package's GPU operators.

Each window of the spectrum is mapped by a Chebyshev-Jackson filter p to the top
of p(H)'s spectrum and the filtered TRLM finds n_mode eigenpairs there, so the
device holds one Lanczos workspace whatever the total number of modes:

  bound     (PlusI, Lanczos upper bound + 1e-12)                 (lines 182-188)
  window 1  wanted (PlusI, upper / 10), filter fitted by KPM counts to about
            (W - 5) * 5 eigenvalues (margin 25), rigid modes pushed off with a
            Hotelling shift of -40 after the filter              (lines 235-258, 296-323)
  window i  wanted (left, left + 3 * guess), fitted to about W - 5 eigenvalues
            (margin 5), no deflation                             (lines 260-282)
  keep      eigenvalues above the window's left edge; next left edge
            max(eigenvalues) - 1e-10, next guess |last - first|  (lines 325, 341-346, 368)
  files     per window Eigval_/PerformanceList_InchingManyCTRLM_..._<offset>.pkl
            and resume from them                                 (lines 16-38, 347-350, 399-415)

Difference: a mode that the next window finds again (the reference's left edge
max - 1e-10 admits the previous window's top mode; the notebook leaves the
duplicates in) is dropped when its eigenvector overlaps one of the previous
window's by more than 1/sqrt(2); eigenvalue equality is not used, so exactly
degenerate modes are kept.  The window files hold no eigenvectors, so the first
window after a resume drops values within 1e-9 * ||H|| of the last saved
window's eigenvalues instead.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import results
from .krylov import HessianOperator
from .spectrum import estimate_spectrum_bound, optimize_params_on_memory
from .solvers.trlm import trlm

OVERLAP_DUPLICATE = 2 ** -0.5


def ctrlm_many_modes(H, total_modes, n_mode=28, Q=None, tol=1e-12, maxiter=15000, wanted_number=None,
                     max_degree=5120, min_degree=5, kpm_trials=5, hotelling_shift=-40.0, precision="f64",
                     seed=0, checkpoint=None, on_window=None, keep_vectors=False, max_windows=1000,
                     verbose=False):
    """Lowest total_modes non-rigid modes of the store H, window by window.

    Q: rigid-body basis (rows), deflated in the first window only.
    checkpoint: dict(folder, pdbid, platform, device[, pdbfn, n_atoms,
    maxleafsize]) -> window files are written, and an interrupted march resumes
    from them.  on_window(eigval, eigvec) receives each window's kept modes
    (eigenvalues incl. PlusI, eigenvectors (n, m) on the device).  With
    keep_vectors, the kept eigenvectors are also collected on the host.

    Returns dict(eigvals (PlusI removed, ascending, numpy), residuals
    ||H v - lambda v|| (numpy), windows (list of dicts), eigvecs (n, m) numpy or None)."""
    assert total_modes > 0 and n_mode > 5, "ABORTED. total_modes > 0 and n_mode > 5 are required"
    plus_i = float(H.plus_i)
    W = int(wanted_number or n_mode)
    op64 = HessianOperator(H, prec=64)
    lo_b, hi_b = estimate_spectrum_bound(H, steps=300, seed=seed, precision=precision)
    bound = (plus_i, hi_b + 1e-12)
    state = None
    if checkpoint is not None:
        state = results.load_progress(checkpoint["folder"], checkpoint["pdbid"], checkpoint["platform"],
                                      checkpoint["device"], total_modes, plus_i)
    last_saved = None
    if state is None:
        left, guess, culm, remaining, offset, first = bound[0], 0.25, 0.0, int(total_modes), 0, True
    else:
        left, guess, culm = state["left_bound"], state["interval_guess"], state["cumulative_runtime"]
        remaining, offset, first = state["remaining"], state["next_offset"], False
        last_saved = state["last_eigvals"]
    t0 = time.perf_counter()
    all_ev, all_res, all_vec, windows = [], [], [], []
    prev = None
    while remaining > 0 and len(windows) < max_windows:
        tw = time.perf_counter()
        common = dict(User_MaximumDegree=max_degree, User_MinimumDegree=min_degree, User_DampingKernel="Jackson",
                      User_ExtremalIntervalDefinition=1e-10, User_SpectrumBound=bound, User_NumberKpmTrials=kpm_trials,
                      User_ConvergenceRatio=0.7, precision=precision, seed=seed + len(windows))
        if first:
            pol, count, interval = optimize_params_on_memory(
                H, User_WantedInterval=(plus_i, bound[1] / 10), User_DesignatedStart=bound[1] / 10,
                User_WantedNumberEigenvalue=(W - 5) * 5, User_AffordableMemoryMargin=25, **common)
        else:
            pol, count, interval = optimize_params_on_memory(
                H, User_WantedInterval=(left, left + 3.0 * guess), User_DesignatedStart=left + 3.0 * guess,
                User_WantedNumberEigenvalue=W - 5, User_AffordableMemoryMargin=5, **common)
        ev, V, info = trlm(H, k=n_mode, tol=tol, maxiter=maxiter, workspace_factor=2, Q=Q if first else None,
                           shift=hotelling_shift, polynomial=pol, precision=precision, seed=seed + len(windows),
                           return_info=True)
        evn = ev.cpu().numpy()
        guess = float(abs(evn[-1] - evn[0]))
        keep = evn > interval[0]
        if prev is not None and keep.any():
            ov = (prev.t() @ V).abs().max(dim=0).values.cpu().numpy()
            keep &= ov <= OVERLAP_DUPLICATE
        elif last_saved is not None and keep.any():
            gap = np.abs(evn[:, None] - last_saved[None, :]).min(axis=1)
            keep &= gap > 1e-9 * bound[1]
        idx = np.nonzero(keep)[0]
        idx_t = torch.from_numpy(idx).to(V.device)
        evk, Vk = ev[idx_t], V[:, idx_t].contiguous()
        if len(idx):
            R = op64(Vk) - Vk * evk[None, :]
            res = torch.linalg.vector_norm(R, dim=0).cpu().numpy()
        else:
            res = np.zeros(0)
        seconds = time.perf_counter() - tw
        win = dict(interval=tuple(float(x) for x in interval), degree=int(pol.AdjustedDegree), kpm_count=int(count),
                   returned=int(len(evn)), kept=int(len(idx)), offset=int(offset), seconds=seconds,
                   trlm_iterations=info["iterations"], trlm_converged=info["converged"], deflated=first)
        windows.append(win)
        if verbose:
            print(f"ctrlm window {len(windows)}: {win}")
        if checkpoint is not None and len(idx):
            results.save_window(checkpoint["folder"], checkpoint["pdbid"], checkpoint["platform"],
                                checkpoint["device"], offset, evk.cpu().numpy() - plus_i, res, pol.AdjustedDegree,
                                pdbfn=checkpoint.get("pdbfn", ""), n_atoms=checkpoint.get("n_atoms", H.n_atoms),
                                runtime=culm + time.perf_counter() - t0,
                                peak_mem_mib=torch.cuda.max_memory_allocated() / 2 ** 20,
                                maxleafsize=checkpoint.get("maxleafsize", 100))
        if on_window is not None and len(idx):
            on_window(evk, Vk)
        all_ev.append(evk.cpu().numpy())
        all_res.append(res)
        if keep_vectors:
            all_vec.append(Vk.cpu().numpy())
        left = float(np.max(evn)) - 1e-10
        prev = V
        remaining -= len(idx)
        offset += len(idx)
        first = False
    ev_all = np.concatenate(all_ev) if all_ev else np.zeros(0)
    order = np.argsort(ev_all)
    out = dict(eigvals=ev_all[order] - plus_i, residuals=(np.concatenate(all_res) if all_res else np.zeros(0))[order],
               windows=windows, seconds=time.perf_counter() - t0, complete=remaining <= 0)
    out["eigvecs"] = np.concatenate(all_vec, axis=1)[:, order] if (keep_vectors and all_vec) else None
    return out
