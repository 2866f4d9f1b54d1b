"""CPU oracle of the ASOHF particle hot path (test infrastructure only)."""
