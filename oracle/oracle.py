"""CPU oracle of PeriDyn's per-step force path -- TEST INFRASTRUCTURE ONLY.

The checker the CUDA library is compared against.  Only tests/,
__graft_entry__.smoke() and the CPU-baseline / reference arm of bench.py
use it; the product library never loads it.

The heavy loops are the C restatement in pd_oracle.c; this module restates
the surrounding reference code (environment assembly, update_acc!, the
velocity-Verlet step, boundary conditions, QSDrag, contact neighbour
updates, damage) with numpy, whose elementwise + and * round exactly like
Julia's unfused Float64 broadcasting.  It consumes the same description
objects as the product (peridyn_b200 materials, contacts, BCs).

Parity status: Julia is not available here and the reference ships no
tests or golden vectors, so this restatement is pinned by analytical
known-answer tests (tests/test_oracle_known_answers.py), not by reference
outputs ("parity unpinned" by the reference itself).
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liborpd.so")

c_dp = ctypes.POINTER(ctypes.c_double)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_u8p = ctypes.POINTER(ctypes.c_uint8)
I64 = ctypes.c_int64
D = ctypes.c_double

_SIG = {
    "or_fld": (D, [D, D]),
    "or_pow": (D, [D, D]),
    "or_cal_family": (ctypes.c_int, [I64, c_dp, D, I64, c_i64p, c_i64p]),
    "or_weighted_volume": (None, [I64, c_dp, c_dp, I64, c_i64p, c_dp]),
    "or_dilatation": (None, [I64, c_dp, c_dp, c_u8p, c_i64p, I64, c_dp, c_dp, c_dp, ctypes.c_int]),
    "or_force_density_T": (None, [ctypes.c_int, I64, I64, c_dp, c_dp, c_dp, c_i64p, c_u8p, c_i64p, I64, c_dp, c_dp,
                                  c_dp, c_dp, c_dp, c_dp, c_dp, c_dp, ctypes.c_int]),
    "or_isapprox_rigid": (ctypes.c_int, [I64, c_dp, c_dp]),
    "or_td_norm2": (None, [I64, I64, c_dp, c_dp, c_i64p, c_u8p, c_i64p, I64, c_dp, c_dp, c_dp, c_dp, c_dp, c_dp,
                           c_dp]),
    "or_force_density_ep": (None, [I64, I64, c_dp, c_dp, c_dp, c_i64p, c_u8p, c_i64p, I64, c_dp, c_dp, c_dp, c_dp,
                                   c_dp, c_dp, c_dp, c_dp, c_dp, c_dp]),
    "or_contact12_neighs": (None, [I64, c_dp, I64, c_dp, D, I64, c_i64p]),
    "or_contact12_force": (None, [I64, I64, c_i64p, c_dp, c_dp, c_dp, c_dp, c_dp, c_dp, c_dp, c_dp, D, D, D]),
    "or_contact11_neighs": (None, [I64, c_dp, I64, c_i64p, c_u8p, D, D, I64, I64, c_i64p]),
    "or_contact11_neighs_ordered": (None, [I64, c_dp, I64, c_i64p, c_u8p, D, D, I64, I64, c_i64p]),
    "or_contact11_force": (None, [I64, I64, c_i64p, c_dp, c_dp, c_dp, c_dp, D, D, D]),
}

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(_HERE, "pd_oracle.c")):
            build()
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIG.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(c_dp)


def _i(a):
    return None if a is None else a.ctypes.data_as(c_i64p)


def _u(a):
    return None if a is None else a.ctypes.data_as(c_u8p)


PMB, LPS, SKIP, EP = 0, 1, 2, 3


def cal_family(x, horizon, max_neigh):
    """peri.jl:571-576 + general_material.jl:85-90: (family, intact)."""
    x = np.asfortranarray(x, dtype=np.float64)
    n = x.shape[1]
    mn = min(max_neigh, n)
    buf = np.zeros(mn * n, dtype=np.int64)
    rows = ctypes.c_int64()
    rc = lib().or_cal_family(n, _d(x), float(horizon), int(max_neigh), _i(buf), ctypes.byref(rows))
    if rc != 0:
        raise IndexError("family exceeds max_neigh (reference: BoundsError)")
    r = rows.value
    fam = np.asfortranarray(buf[: r * n].reshape((r, n), order="F"))
    return fam, fam > 0


def weighted_volume(x, vol, family):
    m = np.zeros(x.shape[1])
    lib().or_weighted_volume(x.shape[1], _d(x), _d(vol), family.shape[0], _i(family), _d(m))
    return m


class _Block:
    pass


class OracleEnv:
    """Mirror of GeneralEnvironment + the reference solver functions."""

    def __init__(self, materials, contacts, bcs, dt, nthreads=1, families=None):
        self.dt = float(dt)
        self.nthreads = int(nthreads)
        self.time_step = 0
        self.blocks = []
        off = 0
        ys, vs, vols, types, bids, masses = [], [], [], [], [], []
        for b, mat in enumerate(materials):
            gen, spc = mat.general, mat.specific
            B = _Block()
            B.mat = mat
            B.kind = spc.kind
            B.n = gen.n
            B.off = off
            B.x = np.asfortranarray(gen.x)
            B.vol = np.ascontiguousarray(gen.volume)
            B.type_start = mat.type.start
            B.nt = len(mat.type)
            B.type_rel = np.ascontiguousarray(gen.type - B.type_start + 1, dtype=np.int64)
            B.density = np.ascontiguousarray(spc.density[: B.nt], dtype=np.float64)
            B.cs = np.asfortranarray(spc.critical_stretch, dtype=np.float64)
            B.c = np.asfortranarray(getattr(spc, "bond_stiffness", np.zeros((B.nt, B.nt))), dtype=np.float64)
            B.K = np.asfortranarray(getattr(spc, "bulk_modulus", np.zeros((B.nt, B.nt))), dtype=np.float64)
            B.G = np.asfortranarray(getattr(spc, "shear_modulus", np.zeros((B.nt, B.nt))), dtype=np.float64)
            if families is not None and families[b] is not None:
                fam, intact = families[b]
                B.family = np.asfortranarray(fam, dtype=np.int64)
                B.intact = np.asfortranarray(fam > 0 if intact is None else (np.asarray(intact) & (fam > 0)),
                                             dtype=np.uint8)
            elif B.kind == SKIP:
                B.family = np.zeros((1, B.n), dtype=np.int64, order="F")
                B.intact = np.zeros((1, B.n), dtype=np.uint8, order="F")
            else:
                fam, intact = cal_family(B.x, gen.horizon, gen.max_neigh)
                B.family = fam
                B.intact = np.asfortranarray(intact, dtype=np.uint8)
            B.m = weighted_volume(B.x, B.vol, B.family)
            B.theta = np.zeros(B.n)
            if B.kind == EP:  # elasto_plastic.jl:60-68 init
                B.psi = np.asfortranarray(spc.psi, dtype=np.float64)
                B.edp = np.zeros(B.family.shape, order="F")
                B.td_norm2 = np.zeros(B.n)
            B.deformed = bool(gen.deformed[0])
            self.blocks.append(B)
            ys.append(gen.y)
            vs.append(gen.velocity)
            vols.append(gen.volume)
            types.append(gen.type)
            bids.append(np.full(B.n, mat.blockid))
            # environment.jl:173-180: mass = volume .* density[type]
            masses.append(gen.volume * B.density[B.type_rel - 1])
            off += B.n
        self.N = off
        self.y = np.asfortranarray(np.hstack(ys))
        self.v = np.asfortranarray(np.hstack(vs))
        self.f = np.zeros((3, self.N), order="F")
        self.p = np.zeros((3, self.N), order="F")
        self.volume = np.concatenate(vols)
        self.type = np.concatenate(types)
        self.bid = np.concatenate(bids)
        self.mass = np.concatenate(masses)
        self.density = self.mass / self.volume  # environment.jl:214
        self.intact0 = np.concatenate([B.intact.sum(axis=0) for B in self.blocks]).astype(np.int64)
        by_id = {id(B.mat): B for B in self.blocks}
        self.contacts = []
        for cm in contacts:
            C = _Block()
            C.model = cm
            C.b1 = by_id[id(cm.mat1)]
            if cm.kind == 0:
                C.b2 = by_id[id(cm.mat2)]
                C.rows = cm.max_neighs
            else:
                C.b2 = C.b1
                C.rows = cm.rows
            C.neighs = np.zeros((C.rows, C.b1.n), dtype=np.int64, order="F")
            self.contacts.append(C)
        self.bcs = []
        for bc in bcs:
            Bc = _Block()
            Bc.kind = bc.kind
            Bc.mask = np.asarray(bc.bool, dtype=bool)
            Bc.dims = np.asarray(bc.dims, dtype=bool)
            Bc.rate = np.asarray(bc.rate, dtype=np.float64)
            Bc.freq = float(bc.freq)
            Bc.applyafter = int(bc.applyafter)
            Bc.onlyatstart = bool(bc.onlyatstart)
            Bc.direction = 1
            Bc.last = np.zeros((3, int(Bc.mask.sum())), order="F")
            Bc.scale = np.asarray(getattr(bc, "scale", np.zeros(3)), dtype=np.float64)
            Bc.fixpoint = np.asarray(getattr(bc, "fixpoint", np.zeros(3)), dtype=np.float64)
            Bc.wait = int(getattr(bc, "wait", 1))
            sb = getattr(bc, "scalebool", None)
            Bc.smask = None if sb is None else np.asarray(sb, dtype=bool)
            Bc.limits = getattr(bc, "limits", None)
            self.bcs.append(Bc)

    # ---------------------------------------------------------------- forces
    def _slice(self, B):
        return slice(B.off, B.off + B.n)

    def force_density_T(self, B):
        """general_material.jl:296-369 (+ out_of_loop!)."""
        if B.kind == SKIP:
            return
        s = self._slice(B)
        y_ = self.y[:, s]
        f_ = self.f[:, s]
        assert y_.flags.f_contiguous and f_.flags.f_contiguous
        M = B.family.shape[0]
        if B.kind in (LPS, EP):
            lib().or_dilatation(B.n, _d(y_), _d(B.x), _u(B.intact), _i(B.family), M, _d(B.vol), _d(B.m),
                                _d(B.theta), self.nthreads)
        if B.kind == EP:  # elasto_plastic.jl:166-172 out_of_loop!, then the bond loop
            lib().or_td_norm2(B.n, M, _d(y_), _d(B.x), _i(B.family), _u(B.intact), _i(B.type_rel), B.nt,
                              _d(B.cs), _d(B.vol), _d(B.m), _d(B.theta), _d(B.G), _d(B.edp), _d(B.td_norm2))
            lib().or_force_density_ep(B.n, M, _d(f_), _d(y_), _d(B.x), _i(B.family), _u(B.intact),
                                      _i(B.type_rel), B.nt, _d(B.cs), _d(B.density), _d(B.vol), _d(B.m),
                                      _d(B.theta), _d(B.K), _d(B.G), _d(B.psi), _d(B.td_norm2), _d(B.edp))
            return
        lib().or_force_density_T(B.kind, B.n, M, _d(f_), _d(y_), _d(B.x), _i(B.family), _u(B.intact),
                                 _i(B.type_rel), B.nt, _d(B.cs), _d(B.density), _d(B.vol), _d(B.c), _d(B.m),
                                 _d(B.theta), _d(B.K), _d(B.G), self.nthreads)

    def force_density(self, B):
        """general_material.jl:240-256 (the deformed gate); skip_specific.jl:62-64."""
        if B.kind == SKIP:
            return
        if B.deformed:
            self.force_density_T(B)
            return
        y_ = np.asfortranarray(self.y[:, self._slice(B)])
        if lib().or_isapprox_rigid(B.n, _d(y_), _d(B.x)):
            return
        B.deformed = True
        self.force_density_T(B)

    def short_range_contact(self, C):
        cm = C.model
        s1 = self._slice(C.b1)
        if cm.kind == 0:  # contacts.jl:210-247
            s2 = self._slice(C.b2)
            f1, f2 = self.f[:, s1], self.f[:, s2]
            lib().or_contact12_force(C.b1.n, C.rows, _i(C.neighs), _d(self.y[:, s1]), _d(self.y[:, s2]), _d(f1),
                                     _d(f2), _d(np.ascontiguousarray(self.volume[s1])),
                                     _d(np.ascontiguousarray(self.volume[s2])),
                                     _d(np.ascontiguousarray(self.density[s1])),
                                     _d(np.ascontiguousarray(self.density[s2])), cm.equi_dist, cm.exponent,
                                     cm.stifness)
        else:  # contacts.jl:357-381
            f1 = self.f[:, s1]
            lib().or_contact11_force(C.b1.n, C.rows, _i(C.neighs), _d(self.y[:, s1]), _d(f1),
                                     _d(np.ascontiguousarray(self.volume[s1])),
                                     _d(np.ascontiguousarray(self.density[s1])), cm.equi_dist, cm.exponent,
                                     cm.stifness)

    def update_acc(self):
        """solvers.jl:320-336."""
        self.f[:] = 0.0
        for B in self.blocks:
            self.force_density(B)
        for C in self.contacts:
            self.short_range_contact(C)
        self.p[:] = self.mass * self.v  # update_misc!

    def update_neighs(self, max_part=30):
        """solvers.jl:351-361 / contacts.jl:434-476, 591-605."""
        for C in self.contacts:
            cm = C.model
            s1 = self._slice(C.b1)
            if cm.kind == 0:
                s2 = self._slice(C.b2)
                x11 = np.asfortranarray(self.y[:, s1])
                x22 = np.asfortranarray(self.y[:, s2])
                lib().or_contact12_neighs(C.b1.n, _d(x11), C.b2.n, _d(x22), cm.distance, C.rows, _i(C.neighs))
            else:
                B = C.b1
                x = np.asfortranarray(self.y[:, s1])
                search = lib().or_contact11_neighs_ordered if getattr(cm, "ordered", False) else \
                    lib().or_contact11_neighs
                search(B.n, _d(x), B.family.shape[0], _i(B.family), _u(B.intact), cm.distance, cm.equi_dist,
                       int(max_part), C.rows, _i(C.neighs))

    # --------------------------------------------------------------- BCs
    def apply_bc_at0(self):
        """FixBC.jl:63 / ToFroBC.jl:94 / DeltaScaleBC.jl:71 /
        ScaleFixWaitBC.jl:80: BC.last .= y[dims, bool]; ContainerBC.jl:84
        does nothing."""
        for bc in self.bcs:
            if bc.kind == 4:
                continue
            for d in range(3):
                if bc.dims[d]:
                    bc.last[d] = self.y[d, bc.mask]

    def _bc_pos(self, bc):
        if bc.kind == 4:  # ContainerBC.jl:58-61: y unchanged
            return
        if bc.kind in (0, 3):  # FixBC.jl:213, ScaleFixWaitBC.jl:59
            new = bc.last
        elif bc.kind == 2:  # DeltaScaleBC.jl:52-55
            g = 1.0 + (bc.scale * self.dt) * float(self.time_step)
            new = (bc.last - bc.fixpoint.reshape(3, 1)) * g.reshape(3, 1) + bc.fixpoint.reshape(3, 1)
        else:  # ToFroBC.jl:286-289
            new = bc.last + (self.dt * bc.direction * bc.rate).reshape(3, 1)
        idx = np.nonzero(bc.mask)[0]
        for d in range(3):
            if bc.dims[d]:
                self.y[d, idx] = new[d]
        if bc.kind == 1:
            for d in range(3):
                if bc.dims[d]:
                    bc.last[d] = new[d]

    def _bc_vel(self, bc):
        idx = np.nonzero(bc.mask)[0]
        if bc.kind == 4:  # ContainerBC.jl:63-68
            if bc.limits is None:
                return
            out = np.zeros(idx.size, dtype=bool)
            for d in range(3):
                if bc.dims[d]:
                    yd = self.y[d, idx]
                    out |= (yd < bc.limits[d, 0]) | (yd > bc.limits[d, 1])
            for d in range(3):
                if bc.dims[d]:
                    self.v[d, idx[out]] = 0.0
            return
        for d in range(3):
            if bc.dims[d]:
                self.v[d, idx] = float(bc.direction) * bc.rate[d] if bc.kind == 1 else 0.0

    def _bc_check(self):
        for bc in self.bcs:
            if bc.kind == 3 and self.time_step % bc.wait == 0:  # ScaleFixWaitBC.jl:63-68
                sidx = np.nonzero(bc.smask)[0]
                for d in range(3):
                    if bc.dims[d]:
                        g = math.sqrt(1.0 + (2.0 * bc.scale[d]) * self.dt)
                        self.y[d, sidx] = (self.y[d, sidx] - bc.fixpoint[d]) * g + bc.fixpoint[d]
                for d in range(3):
                    if bc.dims[d]:
                        bc.last[d] = self.y[d, bc.mask]
            if bc.kind == 1 and (self.time_step > bc.applyafter) and math.fmod(self.time_step, bc.freq) == 0:
                bc.direction = -bc.direction

    # ------------------------------------------------------------ solvers
    def vv_step(self):
        """velocity_verlet.jl:57-89."""
        c = self.dt / 2
        dt = self.dt
        self.v += c * self.f
        self.y += dt * self.v
        for bc in self.bcs:
            self._bc_pos(bc)
        self.update_acc()
        self.v += c * self.f
        for bc in self.bcs:
            self._bc_vel(bc)
        self._bc_check()
        self.time_step += 1

    def minimize(self, step_size, drag, max_iter=1000, x_tol=1e-3, f_tol=1e-3):
        """minimize.jl:105-231; returns the iteration count."""
        for bc in self.bcs:
            self._bc_pos(bc)
            self._bc_vel(bc)
        ps = self.blocks[0].mat.general.particle_size
        mask = np.zeros(self.N, dtype=bool)
        for bc in self.bcs:
            if not bc.onlyatstart:
                mask |= bc.mask
        mask = ~mask
        opt = np.zeros((3, int(mask.sum())), order="F")
        lam = drag
        k = lam / 10
        a = ps / 10
        it = 0
        for i in range(1, max_iter + 1):
            it = i
            self.update_acc()
            gs = self.f[:, mask]
            force = gs - lam * opt * (1.0 + k * np.abs(opt))
            dy = 0.5 * force * (step_size * step_size) + opt * step_size
            opt += step_size * force
            dy = np.maximum(np.minimum(dy, a), -a)
            self.y[:, mask] += dy
            f_tol_ = np.max(np.abs(gs)) if gs.size else 0.0
            x_tol_ = np.max(np.abs(dy)) if dy.size else 0.0
            if (f_tol_ < f_tol) and (x_tol_ < x_tol):
                break
        self._bc_check()
        self.time_step += 1
        return it

    # -------------------------------------------------------- diagnostics
    def damage(self):
        """peri.jl:587-594."""
        intact = np.concatenate([B.intact.sum(axis=0) for B in self.blocks])
        with np.errstate(invalid="ignore", divide="ignore"):
            return 1 - intact / self.intact0

    def run(self, N, filewrite_freq=10, neigh_update_freq=1, start_at=0, write_from=0, max_part=30):
        """solvers.jl:97-187 cadence (file writes = force evaluations)."""
        self.update_acc()  # "start_with"
        self.update_neighs(max_part)
        if start_at == 0:
            self.apply_bc_at0()
        self.update_acc()  # step 0 file
        for i in range(1 + start_at, N + start_at + 1):
            self.vv_step()
            if i % filewrite_freq == 0 or (i == 1 and write_from == 0):
                self.update_acc()
            if i % neigh_update_freq == 0:
                self.update_neighs(max_part)
        self.update_acc()  # "end_with"
