"""ORACLE package: CPU oracles used by tests/ only (see oracle.py)."""
