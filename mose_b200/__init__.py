"""mose_b200 -- B200-native (sm_100a) explicit inviscid residual-and-update path
of the MOSE compressible-flow solver, behind a C ABI (include/mose_gpu.h).

    from mose_b200 import Solver, cases
    s = Solver(cases.isentropic_vortex(256, steps=10))
    s.advance(10)
"""
from . import cases
from .solver import MoseError, Solver

__all__ = ["Solver", "MoseError", "cases"]
