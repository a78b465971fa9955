"""CPU oracle (test infrastructure only; never imported by btorch_b200)."""
