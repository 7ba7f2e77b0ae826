"""B200-native staggered-grid Biot poroelastic stepper with CPML.

The compute path is the CUDA library ``lib/libbiot_b200.so`` (C ABI in
``include/biot.h``); this package is its Python host mirror.
"""
from ._abi import FIELDS, PREC, TRACES, BiotError, load  # noqa: F401
from .biot import Batch, Medium, Server, ShotConfig, Simulation  # noqa: F401

__all__ = ["Simulation", "Batch", "Server", "ShotConfig", "Medium", "BiotError", "load", "FIELDS", "TRACES", "PREC"]
