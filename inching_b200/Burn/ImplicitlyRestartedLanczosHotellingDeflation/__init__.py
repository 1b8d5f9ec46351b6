"""Reference-compatible module path (InchingLiteInteger.Burn.ImplicitlyRestartedLanczosHotellingDeflation)."""
