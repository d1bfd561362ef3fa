"""Oracle: CPU checker for the B200 library (test infrastructure only)."""
