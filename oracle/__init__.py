"""CPU oracle for the Redi step — test infrastructure, never the product path."""
