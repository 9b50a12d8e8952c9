"""B200-native walk-on-spheres (placeholder during bring-up)."""
