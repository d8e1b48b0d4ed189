"""CPU oracle for the alignment hot path — test infrastructure only (see oracle.h)."""
