"""CPU oracle for the growth step -- test infrastructure, never the product."""
