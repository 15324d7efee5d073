"""Boundary conditions mirroring src/boundary_conditions/{FixBC,ToFroBC,
DeltaScaleBC,ScaleFixWaitBC,ContainerBC}.jl.

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


class DeltaScaleBC(BoundaryCondition):
    """DeltaScaleBC.jl:47-60: y = (last - fixpoint) * (1 + scale*dt*time_step)
    + fixpoint, v = 0; last is the position at apply_bc_at0."""

    kind = _abi.PD_BC_DELTA_SCALE

    def __init__(self, bool, scale, fixpoint, dims=(True, True, True), onlyatstart=False):
        self.bool = np.ascontiguousarray(np.asarray(bool, dtype=np.uint8).reshape(-1))
        self.dims = np.asarray(list(dims)[:3], dtype=np.uint8)
        self.scale = np.asarray(scale, dtype=np.float64).reshape(-1)[:3].copy()
        self.fixpoint = np.asarray(fixpoint, dtype=np.float64).reshape(-1)[:3].copy()
        self.onlyatstart = bool_(onlyatstart)
        self.rate = np.zeros(3)
        self.freq = math.inf
        self.applyafter = 0


class ScaleFixWaitBC(BoundaryCondition):
    """ScaleFixWaitBC.jl:46-71: y = last, v = 0; at every step with
    time_step % wait == 0 (check!) the ``scalebool`` particles are scaled
    about ``fixpoint`` by sqrt(1 + 2*scale*dt) and last is re-read."""

    kind = _abi.PD_BC_SCALE_FIX_WAIT

    def __init__(self, bool, scale, fixpoint, wait, scalebool, dims=(True, True, True), applyafter=0,
                 onlyatstart=False):
        self.bool = np.ascontiguousarray(np.asarray(bool, dtype=np.uint8).reshape(-1))
        self.scalebool = np.ascontiguousarray(np.asarray(scalebool, dtype=np.uint8).reshape(-1))
        self.dims = np.asarray(list(dims)[:3], dtype=np.uint8)
        self.scale = np.asarray(scale, dtype=np.float64).reshape(-1)[:3].copy()
        self.fixpoint = np.asarray(fixpoint, dtype=np.float64).reshape(-1)[:3].copy()
        self.wait = int(wait)
        self.onlyatstart = bool_(onlyatstart)
        self.rate = np.zeros(3)
        self.freq = math.inf
        self.applyafter = int(applyafter)  # stored, unused (as in the reference)


class ContainerBC(BoundaryCondition):
    """ContainerBC.jl:48-74: zero the velocity (in ``dims``) of particles of
    ``bool`` whose position has left ``limits`` (3x2: lower, upper bounds);
    positions are untouched.  ``limits=None`` does nothing.  (The
    reference's constructor tests an undefined name ``limit``; this follows
    its documented behaviour.)"""

    kind = _abi.PD_BC_CONTAINER

    def __init__(self, bool, limits=None, dims=(True, True, True), onlyatstart=False):
        self.bool = np.ascontiguousarray(np.asarray(bool, dtype=np.uint8).reshape(-1))
        self.dims = np.asarray(list(dims)[:3], dtype=np.uint8)
        self.limits = None if limits is None else np.asfortranarray(np.asarray(limits, dtype=np.float64)[:3, :2])
        self.onlyatstart = bool_(onlyatstart)
        self.rate = np.zeros(3)
        self.freq = math.inf
        self.applyafter = 0


def bool_(v):
    return bool(v)
