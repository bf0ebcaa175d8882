"""CPU oracle for the BN254 hot path (test infrastructure only)."""
