"""B200-native JGS2 elastodynamics step (host-side package)."""
