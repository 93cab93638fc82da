"""CPU oracle of the solver's hot path (test infrastructure only)."""
