"""CPU oracle of the element assembly (test infrastructure only)."""
