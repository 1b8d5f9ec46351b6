"""Reference-compatible module path (InchingLiteInteger.Burn.JacobiDavidsonHotellingDeflation)."""
