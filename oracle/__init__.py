"""Test-only checkers for the B200 kernels (never imported by the product).

  oracle/qs_oracle.c  - C restatement of the reference CPU backend -> _build/liboracle.so
  oracle/_ref/        - the reference's own CPUQuantumGates.cpp compiled from its
                        sources (built here when the reference tree is present)
"""
