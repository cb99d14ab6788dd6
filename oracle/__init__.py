"""CPU oracle for the finite-volume Euler path (test infrastructure only).

Loaded by the tests, by the smoke check and by bench.py's CPU-baseline leg;
never by the product package.  See fvm_oracle.cpp for what it restates.
"""
from .pyoracle import OracleMesh, OracleSolver, load, mesh_arrays  # noqa: F401
