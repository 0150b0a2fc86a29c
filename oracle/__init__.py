"""CPU FP64 oracle for the two-electron integral path (test infrastructure only)."""
