"""su2_b200: the B200 (sm_100a) device path of the su2 Monte-Carlo hot path.

The product is the C ABI in include/su2b.h, implemented by the in-tree libsu2b.so
(su2_b200/csrc, built with ``python -m su2_b200.build``).  This package exposes it to
Python through ctypes with the reference's names (``gaugeconfig`` and its methods).
"""
from ._abi import Su2bError, load  # noqa: F401
from .lattice import (SolveResult, TrajectoryResult, gaugeconfig,  # noqa: F401
                      read_nconf_counter, update_nconf_counter)

__all__ = ["gaugeconfig", "TrajectoryResult", "SolveResult", "Su2bError", "load",
           "read_nconf_counter", "update_nconf_counter"]
