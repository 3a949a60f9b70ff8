"""CPU oracle of the env-map shading path -- test infrastructure only (see oracle.py)."""
