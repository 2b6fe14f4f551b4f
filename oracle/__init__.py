"""CPU oracle of the ROMSPath particle step -- test infrastructure only.

Imported by tests/, the smoke check and bench.py's CPU-baseline leg, never
by the product package.  Parity unpinned against the reference binary
(no tests, golden vectors or Fortran compiler exist for it here).
"""
