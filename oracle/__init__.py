"""Test oracles (test infrastructure only; never imported by phg_b200)."""
