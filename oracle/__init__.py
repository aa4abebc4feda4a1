"""CPU oracle for the meturay_b200 hot path (test infrastructure only)."""
