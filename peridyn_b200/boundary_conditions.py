"""Boundary conditions mirroring src/boundary_conditions/{FixBC,ToFroBC}.jl.

``bool`` is a mask over all particles of the environment the condition is
used in; ``dims`` selects the constrained coordinates.
"""
import math

import numpy as np

from . import _abi


class BoundaryCondition:
    pass


class FixBC(BoundaryCondition):
    """FixBC.jl:46-65: y[dims, bool] = last (snapshot at t0), v = 0."""

    kind = _abi.PD_BC_FIX

    def __init__(self, bool, dims=(True, True, True), onlyatstart=False):
        self.bool = np.ascontiguousarray(np.asarray(bool, dtype=np.uint8).reshape(-1))
        self.dims = np.asarray(list(dims)[:3], dtype=np.uint8)
        self.onlyatstart = bool_(onlyatstart)
        self.rate = np.zeros(3)
        self.freq = math.inf
        self.applyafter = 0


class ToFroBC(BoundaryCondition):
    """ToFroBC.jl:51-111: y = last + dt*direction*rate, v = direction*rate;
    the direction flips when time_step > applyafter and time_step % freq == 0."""

    kind = _abi.PD_BC_TOFRO

    def __init__(self, bool, rate, freq, dims=(True, True, True), applyafter=0, onlyatstart=False):
        self.bool = np.ascontiguousarray(np.asarray(bool, dtype=np.uint8).reshape(-1))
        self.dims = np.asarray(list(dims)[:3], dtype=np.uint8)
        self.rate = np.asarray(rate, dtype=np.float64).reshape(-1)[:3].copy()
        self.freq = float(freq)
        self.applyafter = int(applyafter)
        self.onlyatstart = bool_(onlyatstart)
        self.direction = 1


def MoveBC(bool, rate, **kwargs):
    """ToFroBC.jl:51-53: a ToFroBC that never flips (freq = Inf)."""
    return ToFroBC(bool, rate, math.inf, **kwargs)


def bool_(v):
    return bool(v)
