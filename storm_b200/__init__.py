"""B200-native Implicit Monte Carlo transport engine (STORM hot path)."""
