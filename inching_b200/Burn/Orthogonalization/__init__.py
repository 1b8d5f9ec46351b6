"""Reference-compatible module path (InchingLiteInteger.Burn.Orthogonalization)."""
