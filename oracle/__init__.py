"""CPU oracle of the reference solver (test infrastructure only)."""
