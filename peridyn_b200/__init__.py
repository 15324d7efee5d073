"""peridyn_b200: B200 (sm_100a) implementation of PeriDyn's per-step force
path behind a C ABI (include/peridyn_b200.h, libperidyn_b200.so).

The Python layer mirrors the reference's Julia API (materials, contacts,
boundary conditions, Env, solvers, run!) and sequences device calls; all
arithmetic runs in the CUDA library.
"""
from ._abi import PDError, device_count, lib
from .boundary_conditions import ContainerBC, DeltaScaleBC, FixBC, MoveBC, ScaleFixWaitBC, ToFroBC
from .contacts import (LinearSpringContactModel, NonLinearSpringContactModel, NonLinearSpringContactModel11,
                       NonLinearSpringContactModel12, ShortRangeContactModel)
from .environment import Env, GeneralEnvironment
from .serving import Server, serve_stream
from .materials import (BondBasedMaterial, BondBasedSpecific, ElastoPlasticSolidSpecific, GeneralMaterial,
                        OrdinaryStateBasedMaterial, OrdinaryStateBasedSpecific, PeridynamicsMaterial, SkipMaterial,
                        SkipSpecific, VonMises, julia_pow_int, make_matrix)
from .solvers import (DSVelocityVerlet, QSDrag, apply_bc_at0, apply_solver, cal_damage, minimize, printdata, run,
                      save_state, simulate, update_acc, update_neighs, velocity_verlet_step)

__all__ = [n for n in dir() if not n.startswith("_")]
