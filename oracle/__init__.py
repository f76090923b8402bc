"""CPU oracle for the fluxion solve path (test infrastructure only; see fx_oracle.h)."""
