"""CPU oracle for the MGPoisson2D hot path (test infrastructure only; see mgp_oracle.h)."""
