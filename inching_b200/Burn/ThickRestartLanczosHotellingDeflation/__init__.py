"""Reference-compatible module path (InchingLiteInteger.Burn.ThickRestartLanczosHotellingDeflation)."""
