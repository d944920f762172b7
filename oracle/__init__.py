"""CPU oracle for the solver (test infrastructure only)."""
