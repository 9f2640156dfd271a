"""fosite_b200: B200-native (sm_100a, FP64) backend for fosite's explicit
finite-volume time step, exposed through the C ABI of include/fosite_gpu.h.

Python modules:
  abi       ctypes mirror of the header (config/status structs, constants)
  sim       Simulation: host mirror of fosite's FirstStep/Step/Run sequence
  problems  seeded initial data of the benchmark workloads
  build     nvcc recipe of lib/libfosite_gpu.so (and the --fmad=false variant)
"""
from . import abi  # noqa: F401

__all__ = ["abi", "sim", "problems"]
