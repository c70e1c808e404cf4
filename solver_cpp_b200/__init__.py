"""B200-native Krylov hot path of solver_cpp (placeholder; binding added below)."""
