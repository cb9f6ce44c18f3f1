"""CPU checkers for the B200 Cholesky path (test infrastructure only)."""
