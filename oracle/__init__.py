"""CPU oracle package: TEST INFRASTRUCTURE ONLY (see oracle.py)."""
