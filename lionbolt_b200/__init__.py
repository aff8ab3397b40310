"""B200-native (sm_100a) transport-solve hot path of Lionbolt.

Public surface mirrors src/LionboltAPI.f90: TransportOp, ScatteringOp, BoltzmannOp,
SpaceAngleVector, AngularClass, XSType, plus MultigroupSolver (the group loop of Main.f90) and
BatchSolver (many independent dose problems solved together on one GPU).
The compute path is the CUDA library lionbolt_b200/liblionbolt_b200.so (C ABI in
include/lionbolt_b200.h); there is no CPU fallback.
"""
from ._lib import LionboltError, load, sn_quadrature  # noqa: F401
from .operators import (AngularClass, BatchSolver, BoltzmannOp, MultigroupSolver, ScatteringOp,  # noqa: F401
                        SpaceAngleVector, TransportOp, XSType)
from . import mesh, problems  # noqa: F401

__all__ = ["LionboltError", "load", "sn_quadrature", "AngularClass", "BatchSolver", "BoltzmannOp", "MultigroupSolver",
           "ScatteringOp", "SpaceAngleVector", "TransportOp", "XSType", "mesh", "problems"]
