"""The oracle's Hessian against the reference's own dense Hessian.

tests/golden/hessian_*.npz hold X_D_K_Hessian (InchingLiteInteger/Burn/
Coordinate/T3.py:47-127) run by tests/golden/make_golden.py on two seeded
structures (one with pairs exactly at, one ulp inside and outside the cutoff, a
duplicate and an isolated atom), PlusI = 1, stored as the lower triangle.  The
oracle's restatement of the sparse path (Fuel/T1.py:276-455) must give the same
matrix to 1e-12 of its largest entry (the two differ only in rounding order)."""
import numpy as np
import pytest

from oracle import hessian as oh

TOL = 1e-12
CASES = ["near_cutoff", "globule400"]


def load_dense(name):
    g = np.load(f"tests/golden/hessian_{name}.npz")
    n = int(g["n"])
    L = np.zeros((n, n))
    L[g["rows"], g["cols"]] = g["vals"]
    return g, L + np.tril(L, -1).T


@pytest.mark.parametrize("name", CASES)
def test_oracle_hessian_matches_reference_dense(name):
    g, Href = load_dense(name)
    A, Ad = oh.hessian_lower(g["X"], float(g["rc_nm"]) * 10.0, float(g["plus_i"]))
    H = oh.full_from_lower(A, Ad)
    scale = np.abs(Href).max()
    assert np.abs(H - Href).max() <= TOL * scale
    # the reference's matrix is symmetric and has the six rigid-body motions at PlusI
    Q = oh.rigid_body_basis(g["X"])
    assert np.abs(Href @ Q.T - float(g["plus_i"]) * Q.T).max() <= 1e-10 * scale
