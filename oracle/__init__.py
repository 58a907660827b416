"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the force path (see oracle.py)."""
