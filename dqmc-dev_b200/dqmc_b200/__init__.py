"""dqmc_b200: B200-native DQMC sweep engine (Python side).

The engine itself is C/CUDA behind the C ABI of include/dqmc_b200.h, built
into lib/libdqmc_b200.so; this package loads that library (failing loudly if
it is absent), reads and writes the DQSF sim-file container, generates sim
files, and binds the gradient path to torch.
"""
from . import simfile  # noqa: F401

__all__ = ["simfile"]
