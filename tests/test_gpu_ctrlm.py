"""Interval-marching filtered TRLM (many modes at constant memory) against dense
LAPACK: every kept mode is an eigenpair (residual <= 1e-8 ||H||), no mode is
kept twice, the march covers the lowest modes without gaps, and a march that
stops early resumes from its window files."""
import numpy as np
import pytest
import torch

from oracle import hessian as oh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glob():
    from inching_b200 import graph, synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    X = synth.globule(1200, seed=9) / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = X[order.cpu().numpy()]
    H = HessianStore(Xr, 8.0, plus_i=1.0)
    A, Ad = oh.hessian_lower(Xr, 8.0, 1.0)
    w = np.linalg.eigvalsh(oh.full_from_lower(A, Ad).toarray())
    return dict(H=H, Q=rigid_body_basis(torch.from_numpy(Xr).cuda()), w=w)


def _check(out, w, total):
    ev = out["eigvals"] + 1.0
    assert len(ev) >= total
    # every kept value is an eigenvalue, and none twice
    j = np.searchsorted(w, ev).clip(1, len(w) - 1)
    near = np.minimum(np.abs(w[j] - ev), np.abs(w[j - 1] - ev))
    assert near.max() < 1e-8 * w[-1]
    assert out["residuals"].max() < 1e-8 * w[-1]
    # the lowest `total` non-rigid modes are all present, none twice
    assert np.abs(np.sort(ev)[:total] - w[6:6 + total]).max() < 1e-8 * w[-1]


def test_ctrlm_march_matches_dense(glob):
    from inching_b200.ctrlm import ctrlm_many_modes
    out = ctrlm_many_modes(glob["H"], 60, n_mode=20, Q=glob["Q"], tol=1e-10, max_degree=2000)
    print("\n", [(round(wd["interval"][0], 3), round(wd["interval"][1], 3), wd["degree"], wd["kept"])
                 for wd in out["windows"]])
    assert out["complete"] and len(out["windows"]) >= 2
    _check(out, glob["w"], 60)


def test_ctrlm_resume_from_window_files(glob, tmp_path):
    from inching_b200.ctrlm import ctrlm_many_modes
    ck = dict(folder=str(tmp_path), pdbid="glob1200", platform="Linux", device="B200")
    first = ctrlm_many_modes(glob["H"], 60, n_mode=20, Q=glob["Q"], tol=1e-10, max_degree=2000, checkpoint=ck,
                             max_windows=1)
    assert not first["complete"]
    rest = ctrlm_many_modes(glob["H"], 60, n_mode=20, Q=glob["Q"], tol=1e-10, max_degree=2000, checkpoint=ck)
    assert rest["complete"] and rest["windows"][0]["offset"] == len(first["eigvals"])
    assert not rest["windows"][0]["deflated"]
    merged = dict(eigvals=np.concatenate([first["eigvals"], rest["eigvals"]]),
                  residuals=np.concatenate([first["residuals"], rest["residuals"]]))
    _check(merged, glob["w"], 60)
