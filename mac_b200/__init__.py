"""B200-native MAC-grid free-surface fluid step (pressure projection and advection)."""
