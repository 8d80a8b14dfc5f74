"""B200-native implementation of SPARC's linear wave time step.

The compute path is libsparc_gpu.so (hand-written CUDA for sm_100a behind
the C ABI of include/sparc_gpu.h); this package is its Python host side.
"""
from . import abi, workloads  # noqa: F401
from .abi import SparcError  # noqa: F401
from .sim import Simulation  # noqa: F401

__all__ = ["Simulation", "SparcError", "abi", "workloads"]
