"""Reference-compatible module path (InchingLiteInteger.Fuel)."""
