"""Reference-compatible module path (InchingLiteInteger.Burn.HermitianLanczos)."""
