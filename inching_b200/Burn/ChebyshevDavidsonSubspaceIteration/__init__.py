"""Reference-compatible module path (InchingLiteInteger.Burn.ChebyshevDavidsonSubspaceIteration)."""
