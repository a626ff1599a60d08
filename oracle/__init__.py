"""CPU oracle of the MISA-MD EAM hot path — test infrastructure only (see oracle.py)."""
