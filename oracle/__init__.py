"""CPU oracle of the BRP4 search path -- test infrastructure only (see oracle.py)."""
