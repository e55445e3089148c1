"""Test oracles for the REMC docking hot path (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this package, and only to check the engine's results; the product never does.

  oracle.fp64 ..... ctypes binding of remc_oracle.c, the FP64 restatement
  oracle.ref ...... ctypes binding of the reference engine's own Replica /
                    Molecule code compiled with ref_harness.cpp (_ref/)
"""
