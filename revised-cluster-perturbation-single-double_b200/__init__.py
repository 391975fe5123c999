"""B200-native SF-CIS / SF-CPS(D-3) hot path (package root)."""
