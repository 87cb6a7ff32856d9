"""Test infrastructure: CPU oracles of the finite-volume RHS path (see oracle/oracle.py)."""
