"""CPU oracle for the Inching normal-mode hot path.  TEST INFRASTRUCTURE ONLY.

This package restates the reference algorithms (jhmlam/Inching,
InchingLiteInteger) in plain numpy/scipy so that the CUDA path can be checked
against them.  Only the test-suite, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` may import it, and only as a checker or as the
timed CPU baseline; the product (``inching_b200``) never imports it and has no
CPU fallback.

Pinning (how the oracle itself is validated):
  * neighbours, degrees, Cuthill-McKee order, batch heads and band slices are
    pinned bit-exactly against golden fixtures produced by running the
    reference's own functions (``tests/golden/make_golden.py``);
  * the Hessian, the Krylov operator and the eigensolvers cannot run here (the
    reference needs CuPy/cuSPARSE), so they are restated line by line and
    pinned by known answers instead: symmetry, the six rigid-body null vectors
    (H q = PlusI q), and agreement with dense LAPACK ``eigh`` / ARPACK
    ``eigsh``.  Solver *bits* are parity-unpinned (the reference draws its
    start vector from CuPy's RNG); solver outputs are compared by eigenvalue,
    subspace angle and residual.
"""
