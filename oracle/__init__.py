"""CPU oracle and reference harness: test infrastructure only (see oracle.h)."""
