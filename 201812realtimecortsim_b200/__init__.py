"""B200-native engine for DPSNN's per-timestep LIFCA loop."""
