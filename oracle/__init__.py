"""CPU oracle of the pybrown_b200 parity tests (test infrastructure only)."""
