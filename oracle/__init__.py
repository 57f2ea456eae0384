"""CPU oracle for the MLS-MPM step (test infrastructure only; see oracle.h)."""
