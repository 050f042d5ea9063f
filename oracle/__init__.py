"""CPU oracle for the bounding path (test infrastructure only)."""
