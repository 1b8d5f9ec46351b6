"""Drop-in for InchingLiteInteger.Burn.Krylov.T3: the Krylov matrix-vector
operator factories (Krylov/T3.py:54-239).  Both return ``aux(A, v, u)`` that
writes u = H v in place; the half/full storage distinction of the reference does
not exist here (one full rank-one store, one fused SpMM), so both factories
build the same operator.  ``A_diag`` is accepted for signature compatibility."""
from __future__ import annotations

from ...krylov import HessianOperator


def _factory(A, A_diag=None, precision="f64"):
    op = HessianOperator(A, prec=32 if precision == "mixed" else 64)

    def aux(A_, v, u):
        assert A_ is A, "ABORTED. the operator was built for another matrix"
        op(v, out=u)
        return None

    return aux


def OOC2_HalfMemS_v_KrylovAv_VOID(A, A_diag, precision="f64"):
    return _factory(A, A_diag, precision)


def OOC2_FullMemS_v_KrylovAv_VOID(A, A_diag, precision="f64"):
    return _factory(A, A_diag, precision)
