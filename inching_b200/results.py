"""Result files in the reference's formats, so its downstream tools (mode
visualisation, movie writer, benchmark tables) read this package's output
unchanged.

Formats (pickle protocol 4), as written by the reference's benchmark drivers
(Command8A/commandBenchmark_InchingTRLMHD_Linux_Pdb_0064_A100.py:206-208, 410-423,
470-491) and the many-mode notebook (Notebook/Application/
04_Inching_EigenproblemManyCTRLM.ipynb, driver cell lines 19-38, 347-350, 399-415):

  Eigval_Inching<TAG>_<pdbid>_<platform>_<device>.pkl
      numpy (k,) eigenvalues with PlusI removed, ascending
  Eigvec_Inching<TAG>_<pdbid>_<platform>_<device>.pkl
      numpy (k, N, 3) eigenvectors in the input atom order
  PerformanceList_Inching<TAG>_<pdbid>_<platform>_<device>.pkl
      list of rows [label, structure file, n_atoms, runtime s, peak memory MiB,
                    platform, device, maxleafsize, mode index,
                    ||H v - lambda v|| (with PlusI), eigenvalue - PlusI]
  many-mode windows: the same names for TAG = ManyCTRLM with a trailing
      _<offset> (modes found before the window); the rows carry two more
      fields, the filter degree and the offset.

<device> is the CUDA device name with spaces removed; a driver skips a structure
whose PerformanceList file exists (checkpoint / resume).
"""
from __future__ import annotations

import os
import pickle
import platform as _platform

import numpy as np


def device_label(device_index=0):
    """(platform, device name) as the drivers spell them."""
    import torch
    return _platform.system(), torch.cuda.get_device_name(device_index)


def _name(folder, kind, tag, pdbid, plat, device, offset=None):
    tail = "" if offset is None else f"_{int(offset)}"
    return os.path.join(folder, f"{kind}_Inching{tag}_{pdbid}_{plat}_{device.replace(' ', '')}{tail}.pkl")


def result_exists(folder, tag, pdbid, plat, device, offset=None):
    return os.path.exists(_name(folder, "PerformanceList", tag, pdbid, plat, device, offset))


def _dump(path, obj):
    with open(path, "wb") as fn:
        pickle.dump(obj, fn, protocol=4)


def performance_rows(label, pdbfn, n_atoms, runtime, peak_mem_mib, plat, device, maxleafsize, residuals,
                     eigval_minus_plus_i, extra=()):
    head = [label, pdbfn, int(n_atoms), float(runtime), float(peak_mem_mib), plat, device, maxleafsize]
    return [head + [i, float(residuals[i]), float(eigval_minus_plus_i[i])] + list(extra)
            for i in range(len(residuals))]


def save_modes(folder, tag, pdbid, plat, device, eigval_minus_plus_i, modes_k_n_3=None, *, pdbfn="",
               n_atoms=None, runtime=0.0, peak_mem_mib=0.0, maxleafsize=100, residuals=None, label=None):
    """Write the eigenvalue, eigenvector (if given) and performance pickles of one
    structure; returns the paths written."""
    os.makedirs(folder, exist_ok=True)
    ev = np.asarray(eigval_minus_plus_i, dtype=np.float64)
    paths = [_name(folder, "Eigval", tag, pdbid, plat, device)]
    _dump(paths[-1], ev)
    if modes_k_n_3 is not None:
        paths.append(_name(folder, "Eigvec", tag, pdbid, plat, device))
        _dump(paths[-1], np.asarray(modes_k_n_3, dtype=np.float64))
        if n_atoms is None:
            n_atoms = np.asarray(modes_k_n_3).shape[1]
    res = np.zeros(len(ev)) if residuals is None else np.asarray(residuals, dtype=np.float64)
    label = label or f"Inching ({tag} {plat} {device.replace(' GPU', '')})"
    rows = performance_rows(label, pdbfn, n_atoms or 0, runtime, peak_mem_mib, plat, device, maxleafsize, res, ev)
    paths.append(_name(folder, "PerformanceList", tag, pdbid, plat, device))
    _dump(paths[-1], rows)
    return paths


def save_window(folder, pdbid, plat, device, offset, eigval_minus_plus_i, residuals, degree, *, pdbfn="",
                n_atoms=0, runtime=0.0, peak_mem_mib=0.0, maxleafsize=100, tag="ManyCTRLM"):
    """One interval-marching window: Eigval_..._<offset>.pkl and
    PerformanceList_..._<offset>.pkl (rows end with degree, offset)."""
    os.makedirs(folder, exist_ok=True)
    ev = np.asarray(eigval_minus_plus_i, dtype=np.float64)
    _dump(_name(folder, "Eigval", tag, pdbid, plat, device, offset), ev)
    label = f"Inching (CTRLM Interior {plat} {device.replace(' GPU', '')})"
    rows = performance_rows(label, pdbfn, n_atoms, runtime, peak_mem_mib, plat, device, maxleafsize,
                            np.asarray(residuals, dtype=np.float64), ev, extra=(int(degree), int(offset)))
    _dump(_name(folder, "PerformanceList", tag, pdbid, plat, device, offset), rows)


def load_progress(folder, pdbid, plat, device, total_modes, plus_i=1.0, tag="ManyCTRLM"):
    """Resume state of an interval march from its window files (driver cell lines
    16-38): the last window found at offset ii gives the next left bound
    max(eigval + PlusI) - 1e-10, the interval guess |eigval[-1] - eigval[0]|, the
    cumulative runtime and the modes still wanted.  None when nothing was saved."""
    state = None
    for ii in range(int(total_modes)):
        if not os.path.exists(_name(folder, "PerformanceList", tag, pdbid, plat, device, ii)):
            continue
        with open(_name(folder, "Eigval", tag, pdbid, plat, device, ii), "rb") as fn:
            ev = pickle.load(fn)
        with open(_name(folder, "PerformanceList", tag, pdbid, plat, device, ii), "rb") as fn:
            rows = pickle.load(fn)
        state = dict(left_bound=float(np.max(ev + plus_i)) - 1e-10, interval_guess=float(abs(ev[-1] - ev[0])),
                     cumulative_runtime=float(rows[0][3]) if rows else 0.0,
                     remaining=int(total_modes) - (ii + len(ev)), next_offset=ii + len(ev),
                     last_eigvals=np.asarray(ev, dtype=np.float64) + plus_i)
    return state
