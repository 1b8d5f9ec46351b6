"""Reference-compatible module path (InchingLiteInteger.Burn.Krylov)."""
