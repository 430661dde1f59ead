"""CPU oracle of the analysis step (test infrastructure only; see letkf_oracle.py)."""
