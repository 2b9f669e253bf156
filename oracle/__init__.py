"""CPU oracle of the quasi-static layer loop (test infrastructure only)."""
