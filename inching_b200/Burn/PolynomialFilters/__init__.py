"""Reference-compatible module path (InchingLiteInteger.Burn.PolynomialFilters)."""
