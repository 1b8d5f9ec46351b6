"""Generate the golden fixtures in this folder by running the reference's own code.

Run from the repository root with the reference checkout available:

    python tests/golden/make_golden.py /path/to/Inching
    python tests/golden/make_golden.py /path/to/Inching hessian    # dense Hessians only

It imports InchingLiteInteger's k-d-tree Cuthill-McKee ordering, its ungapped
band-slice routine and its Chebyshev filter design (numpy/scipy only; the
unused openmm/mdtraj/matplotlib imports of util.py are stubbed) and stores their
outputs on seeded synthetic inputs as small .npz files.  The "hessian" step runs
the reference's dense torch Hessian (Burn/Coordinate/T3.py) on the CPU.  Nothing at test time
reads the reference; the tests only read these files.
"""
from __future__ import annotations

import contextlib
import io
import os
import sys
import types

import numpy as np
import scipy

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from inching_b200 import synth  # noqa: E402


def _import_reference(ref_root):
    for m in ["openmm", "openmm.app", "mdtraj", "matplotlib", "matplotlib.pyplot"]:
        sys.modules.setdefault(m, types.ModuleType(m))
    sys.path.insert(0, ref_root)
    import InchingLiteInteger.Fuel.Coordinate.T1 as coord          # noqa
    import InchingLiteInteger.Burn.PolynomialFilters.T0 as polyt0  # noqa
    return coord, polyt0


def _quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()), contextlib.redirect_stderr(io.StringIO()):
        return fn(*a, **k)


def _adjacency(X_nm, rc_nm):
    """Neighbour lists exactly as the reference queries them
    (cKDTree.query_ball_point, p=2, eps=0, sorted ascending, self included)."""
    from scipy.spatial import cKDTree
    tree = cKDTree(X_nm)
    nl = tree.query_ball_point(X_nm, rc_nm, p=2.0, eps=0, return_sorted=True)
    deg = np.array([len(v) for v in nl], dtype=np.int32)
    rowptr = np.zeros(len(nl) + 1, dtype=np.int64)
    rowptr[1:] = np.cumsum(deg)
    cols = np.concatenate([np.asarray(v, dtype=np.int32) for v in nl]) if len(nl) else np.zeros(0, np.int32)
    return deg, rowptr, cols


def _slices_to_arrays(d):
    """dict{batch: [(s, e), ...]} -> (counts per batch, flat starts, flat ends)."""
    nb = len(d)
    counts = np.array([len(d[i]) for i in range(nb)], dtype=np.int64)
    starts = np.array([s for i in range(nb) for (s, e) in d[i]], dtype=np.int64)
    ends = np.array([e for i in range(nb) for (s, e) in d[i]], dtype=np.int64)
    return counts, starts, ends


def near_cutoff_structure():
    """Pairs placed exactly at, one ulp inside and one ulp outside the 0.8 nm
    cutoff, a coincident (duplicate) atom and an isolated atom, embedded in a
    small globule."""
    base = synth.globule(300, seed=21) / 10.0
    rc = 8.0 / 10.0
    extra = []
    o = np.array([5.0, 5.0, 5.0])
    extra.append(o)
    extra.append(o + np.array([rc, 0.0, 0.0]))                          # exactly rc
    extra.append(o + np.array([0.0, np.nextafter(rc, 0.0), 0.0]))       # 1 ulp inside
    extra.append(o + np.array([0.0, 0.0, np.nextafter(rc, 1.0)]))       # 1 ulp outside
    extra.append(o.copy())                                              # duplicate of o
    extra.append(np.array([-9.0, -9.0, -9.0]))                          # isolated
    p = np.array([0.3, 0.4, 0.0]) * 1.0
    extra.append(o + p)
    extra.append(o + p + np.array([0.48, 0.64, 0.0]))                   # |d| = 0.8 (rounded)
    X = np.concatenate([base, np.array(extra)], axis=0)
    return X.astype(np.float64)


def main(ref_root):
    coord, polyt0 = _import_reference(ref_root)
    meta = dict(numpy=np.__version__, scipy=scipy.__version__)

    cases = {
        "globule2k": synth.globule(2000, seed=11) / 10.0,
        "two_components": np.concatenate([
            synth.globule(800, seed=12) / 10.0,
            synth.globule(700, seed=13) / 10.0 + np.array([20.0, 0.0, 0.0]),
            np.array([[-30.0, 0.0, 0.0], [0.0, -30.0, 0.0], [0.0, 0.0, -30.0]])]),
        "near_cutoff": near_cutoff_structure(),
        "shuffled1k": synth.globule(1000, seed=14)[np.random.default_rng(5).permutation(1000)] / 10.0,
    }
    for name, X in cases.items():
        X = np.ascontiguousarray(X, dtype=np.float64)
        deg, rowptr, cols = _adjacency(X, 0.8)
        order, undo = _quiet(coord.X_KdCuthillMckeeOrder, X.copy(), rc_Gamma=8.0, Reverse=True)
        Xr = np.ascontiguousarray(X[order])
        sl, halfnnz = _quiet(coord.X_KdUngappedMinMaxNeighbor, Xr.copy(), rc_Gamma=8.0,
                             maxleafsize=100, User_ReturnHalfNnz=True, SliceForm=True)
        c, s, e = _slices_to_arrays(sl)
        # band slices on the un-reordered input too: it has real gaps
        sl0 = _quiet(coord.X_KdUngappedMinMaxNeighbor, X.copy(), rc_Gamma=8.0,
                     maxleafsize=100, User_ReturnHalfNnz=False, SliceForm=True)
        c0, s0, e0 = _slices_to_arrays(sl0)
        np.savez_compressed(
            os.path.join(HERE, f"rcm_{name}.npz"), X=X, degree=deg, rowptr=rowptr, cols=cols,
            seed_order=np.argsort(deg), order=np.asarray(order, np.int64), undo=np.asarray(undo, np.int64),
            slice_counts=c, slice_starts=s, slice_ends=e, halfnnz=np.float64(halfnnz),
            raw_slice_counts=c0, raw_slice_starts=s0, raw_slice_ends=e0, **meta)
        print(name, X.shape[0], "deg", deg.mean(), "slices", len(c), "raw gaps", int((c0 > 1).sum()))

    # config-0 size: ordering only (no adjacency, to keep the file small)
    X = synth.globule(5000, seed=0) / 10.0
    order, undo = _quiet(coord.X_KdCuthillMckeeOrder, X.copy(), rc_Gamma=8.0, Reverse=True)
    Xr = np.ascontiguousarray(X[order])
    sl, halfnnz = _quiet(coord.X_KdUngappedMinMaxNeighbor, Xr.copy(), rc_Gamma=8.0,
                         maxleafsize=100, User_ReturnHalfNnz=True, SliceForm=True)
    c, s, e = _slices_to_arrays(sl)
    deg, _, _ = _adjacency(X, 0.8)
    np.savez_compressed(os.path.join(HERE, "rcm_globule5k.npz"), X=X, degree=deg,
                        seed_order=np.argsort(deg), order=np.asarray(order, np.int64),
                        undo=np.asarray(undo, np.int64), slice_counts=c, slice_starts=s,
                        slice_ends=e, halfnnz=np.float64(halfnnz), **meta)
    print("globule5k", X.shape[0])

    # periodic xy images: the reference's own X_cKDTreePbcXy on a seeded slab whose
    # atoms lie inside the box (so its boundary shortcut changes nothing)
    rng = np.random.default_rng(17)
    box = np.array([3.6, 3.2, 4.0])
    Xs = rng.random((2500, 3)) * box
    pbc = {"RectBox_Xsize": box[0], "RectBox_Ysize": box[1], "RectBox_Zsize": box[2],
           "X": (0.0, box[0]), "Y": (0.0, box[1]), "Z": (0.0, box[2])}
    tree = coord.X_cKDTreePbcXy(Xs, User_DictCharmmGuiPbc=pbc)
    nl = _quiet(tree.query_ball_point, Xs, 0.8)
    deg = np.array([len(v) for v in nl], dtype=np.int32)
    cols = np.concatenate([np.asarray(v, dtype=np.int32) for v in nl])
    np.savez_compressed(os.path.join(HERE, "pbc_slab.npz"), X=Xs, box=box, degree=deg, cols=cols, **meta)
    print("pbc_slab", Xs.shape[0], "deg", deg.mean())

    # Chebyshev filter design (pure numpy in the reference)
    windows = [
        dict(User_WantedInterval=(1.0, 1.05), User_SpectrumBound=(1.0, 120.0)),      # extremal
        dict(User_WantedInterval=(1.0, 2.0), User_SpectrumBound=(0.9, 60.0)),        # extremal
        dict(User_WantedInterval=(36.8, 37.2), User_SpectrumBound=(1.0, 759.0)),     # interior
        dict(User_WantedInterval=(3.0, 5.0), User_SpectrumBound=(1.0, 80.0)),        # interior
    ]
    out = {}
    for t, w in enumerate(windows):
        for conv in (0.1, 0.7):
            for kern in ("Jackson", "LanczosSigma"):
                pol = _quiet(polyt0.OOC0_OptimizePolynomialParamsOnDegree, User_MaximumDegree=600,
                             User_MinimumDegree=10, User_DampingKernel=kern,
                             User_ExtremalIntervalDefinition=1e-9, User_ConvergenceRatio=conv, **w)
                key = f"w{t}_{kern}_{conv}"
                out[key + "_mu"] = np.asarray(pol.AdjustedCoefficients, np.float64)
                out[key + "_deg"] = np.int64(pol.AdjustedDegree)
                out[key + "_scal"] = np.array([pol.cc, pol.dd, pol.theta_a, pol.theta_b,
                                               float(pol.gam)], np.float64)
                out[key + "_args"] = np.array([w["User_WantedInterval"][0], w["User_WantedInterval"][1],
                                               w["User_SpectrumBound"][0], w["User_SpectrumBound"][1],
                                               conv, 600, 10], np.float64)
                out[key + "_kernel"] = np.array(kern)
    np.savez_compressed(os.path.join(HERE, "polyfilter.npz"), **out, **meta)
    print("polyfilter", len(windows) * 4)


def dense_hessian_reference(ref_root, X_nm, rc_nm, plus_i):
    """The reference's dense torch Hessian, X_D_K_Hessian (InchingLiteInteger/Burn/
    Coordinate/T3.py:47-127), on the CPU: D = pairwise distances, Gamma = 1 within
    the cutoff by cKDTree's rule (self included; the reference zeroes the self
    term through nan_to_num), accumulation in float64.  Its arithmetic runs unchanged; only its
    CUDA-only housekeeping is replaced for the CPU: torch.device(0) maps to the CPU,
    TorchMakePrecision sets the default dtype alone (not the CUDA tensor type) and
    TorchEmptyCache does nothing."""
    import torch
    for m in ["openmm", "openmm.app", "mdtraj", "matplotlib", "matplotlib.pyplot"]:
        sys.modules.setdefault(m, types.ModuleType(m))
    sys.path.insert(0, ref_root)
    import InchingLiteInteger.util as rutil                      # noqa
    import InchingLiteInteger.Burn.Coordinate.T3 as dense        # noqa
    saved = (torch.device, rutil.TorchMakePrecision, rutil.TorchEmptyCache, torch.get_default_dtype())
    real_device = torch.device
    try:
        dense.torch.device = lambda *a, **k: real_device("cpu")
        rutil.TorchMakePrecision = lambda Precision="torch.float64": torch.set_default_dtype(
            {"torch.float64": torch.float64, "torch.float32": torch.float32}[str(Precision)])
        rutil.TorchEmptyCache = lambda: None
        Xn = np.ascontiguousarray(X_nm, dtype=np.float64)
        dif = Xn[None, :, :] - Xn[:, None, :]
        d2 = (dif[..., 0] * dif[..., 0] + dif[..., 1] * dif[..., 1]) + dif[..., 2] * dif[..., 2]
        X = torch.from_numpy(Xn)
        D = torch.from_numpy(np.sqrt(d2))
        # the cutoff graph by cKDTree's rule (squared distance in this order, <= rc^2)
        Gamma = torch.from_numpy((d2 <= rc_nm * rc_nm).astype(np.float64))
        H = _quiet(dense.X_D_K_Hessian, X, D, Gamma, maxleafsize=100, PlusI=plus_i, dtype_temp=torch.float64)
    finally:
        torch.device, rutil.TorchMakePrecision, rutil.TorchEmptyCache = saved[:3]
        torch.set_default_dtype(saved[3])
    return H.numpy()


def hessian_goldens(ref_root):
    """Dense reference Hessians on two seeded structures (the edge-case structure of
    near_cutoff_structure and a 400-atom globule), stored as their lower triangle
    (incl. diagonal) in COO form: rows, cols int32, vals float64."""
    meta = dict(numpy=np.__version__, scipy=scipy.__version__)
    import torch
    meta["torch"] = torch.__version__
    cases = {"near_cutoff": near_cutoff_structure(), "globule400": synth.globule(400, seed=31) / 10.0}
    for name, X in cases.items():
        H = dense_hessian_reference(ref_root, X, 0.8, 1.0)
        r, c = np.nonzero(np.tril(H))
        np.savez_compressed(os.path.join(HERE, f"hessian_{name}.npz"), X=X, rc_nm=np.float64(0.8),
                            plus_i=np.float64(1.0), rows=r.astype(np.int32), cols=c.astype(np.int32),
                            vals=H[r, c], n=np.int64(H.shape[0]), **meta)
        print("hessian", name, X.shape[0], "nnz(lower)", len(r))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[2] == "hessian":
        hessian_goldens(sys.argv[1])
        sys.exit(0)
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("INCHING_REFERENCE", "../Inching"))
