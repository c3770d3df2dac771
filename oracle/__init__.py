"""CPU oracle and reference-kernel harness (test and measurement infrastructure only)."""
