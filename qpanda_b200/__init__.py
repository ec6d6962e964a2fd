"""qpanda_b200 - a B200-native state-vector backend for the QPanda gate interface.

The product is the sm_100a CUDA library qpanda_b200/_lib/libqsb200.so with the C
ABI of include/qpanda_b200.h, and the C++ QuantumGates subclass in
qpanda_b200/host/.  This Python package is a thin ctypes view of the C ABI
(used by tests and bench.py) plus seeded workload generators.
"""
from .capi import (GATE_DTYPE, OP, QS_C64, QS_C128, Batch, FusionPlan, QSError, Server,  # noqa: F401
                   StateVector, autotune_batch, autotune_plan, format_outcomes, lib)
from . import circuits  # noqa: F401
