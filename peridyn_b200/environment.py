"""``Env``/``GeneralEnvironment`` mirroring src/environment.jl.

The environment owns a device-resident simulation (a ``pd_env`` of
libperidyn_b200.so).  Host attributes that never change (type, bid, volume,
mass, density, intact0, boundaries) are kept as numpy arrays; the state
(y, v, f, p, time_step) is read from and written to the device on access.
"""
import ctypes

import numpy as np

from . import _abi
from .boundary_conditions import BoundaryCondition
from .contacts import NonLinearSpringContactModel11, NonLinearSpringContactModel12


class GeneralEnvironment:
    def __init__(self, id, materials, short_range_contact, boundary_conds, dt, state=2, bskin=0.5, units=False,
                 precision="fp64_serial", device=0, families=None, finalize=True):
        L = _abi.lib()
        self.id = int(id)
        self.state = int(state)
        self.dt = float(dt)
        self.bskin = float(bskin)
        self.material_blocks = list(materials)
        self.short_range_contact = list(short_range_contact)
        self.boundary_conditions = list(boundary_conds)
        self.precision = precision
        self.Collect = None
        self.Params = {}
        self.Out = {}
        self.cprint = lambda env: None
        prec = _abi.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        h = ctypes.c_void_p()
        _abi.check(L.pd_env_create(ctypes.byref(h), int(device), prec, self.dt))
        self._h = h
        try:
            self._assemble(L, families, finalize)
        except Exception:
            L.pd_env_destroy(self._h)
            self._h = None
            raise

    # ------------------------------------------------------------------
    def _assemble(self, L, families, finalize=True):
        types, bids = [], []
        for b, mat in enumerate(self.material_blocks):
            gen = mat.general
            desc = mat.descriptor()
            out = ctypes.c_int64()
            _abi.check(L.pd_env_add_block(self._h, gen.n, _abi.dptr(gen.x), _abi.dptr(gen.y),
                                          _abi.dptr(gen.velocity), _abi.dptr(gen.volume), _abi.i64ptr(gen.type),
                                          ctypes.byref(desc), ctypes.byref(out)))
            if families is not None and families[b] is not None:
                fam, intact = families[b]
                fam = np.asfortranarray(fam, dtype=np.int64)
                intact = None if intact is None else np.asfortranarray(intact, dtype=np.uint8)
                _abi.check(L.pd_env_set_family(self._h, b, fam.shape[0], _abi.i64ptr(fam), _abi.u8ptr(intact)))
            gen._env, gen._block = self, b
            types.append(gen.type)
            bids.append(np.full(gen.n, mat.blockid, dtype=np.int64))
        self.type = np.concatenate(types)
        self.bid = np.concatenate(bids)
        self.N = self.type.size
        for bc in self.boundary_conditions:
            if not isinstance(bc, BoundaryCondition):
                raise TypeError("boundary_conds must hold FixBC/ToFroBC objects")
            if bc.bool.size != self.N:
                raise ValueError("boundary condition mask must cover every particle of the environment")
            rate = np.ascontiguousarray(bc.rate, dtype=np.float64)
            dims = np.ascontiguousarray(bc.dims, dtype=np.uint8)
            if bc.kind in (_abi.PD_BC_DELTA_SCALE, _abi.PD_BC_SCALE_FIX_WAIT):
                sb = getattr(bc, "scalebool", None)
                if sb is not None and sb.size != self.N:
                    raise ValueError("scalebool must cover every particle of the environment")
                _abi.check(L.pd_env_add_scaled_bc(self._h, bc.kind, _abi.u8ptr(bc.bool), _abi.u8ptr(dims),
                                                  _abi.dptr(bc.scale), _abi.dptr(bc.fixpoint),
                                                  int(getattr(bc, "wait", 1)), _abi.u8ptr(sb),
                                                  int(bc.onlyatstart), None))
            elif bc.kind == _abi.PD_BC_CONTAINER:
                lim = None if bc.limits is None else np.asfortranarray(bc.limits, dtype=np.float64)
                _abi.check(L.pd_env_add_container_bc(self._h, _abi.u8ptr(bc.bool), _abi.u8ptr(dims), _abi.dptr(lim),
                                                     int(bc.onlyatstart), None))
            else:
                _abi.check(L.pd_env_add_bc(self._h, bc.kind, _abi.u8ptr(bc.bool), _abi.u8ptr(dims),
                                           _abi.dptr(rate), bc.freq, bc.applyafter, int(bc.onlyatstart), None))
        blocks = {id(m): b for b, m in enumerate(self.material_blocks)}
        for cm in self.short_range_contact:
            if isinstance(cm, NonLinearSpringContactModel12):
                b1, b2 = blocks[id(cm.mat1)], blocks[id(cm.mat2)]
                rows = cm.max_neighs
            elif isinstance(cm, NonLinearSpringContactModel11):
                b1, b2 = blocks[id(cm.mat1)], -1
                rows = cm.rows
            else:
                raise TypeError("unknown contact model")
            _abi.check(L.pd_env_add_contact(self._h, cm.kind, b1, b2, cm.exponent, cm.stifness, cm.equi_dist,
                                            cm.distance, rows, None))
        if not finalize:  # handed to a Server, which finalizes at admission
            return
        _abi.check(L.pd_env_finalize(self._h))
        self.volume = np.zeros(self.N)
        self.mass = np.zeros(self.N)
        self.density = np.zeros(self.N)
        _abi.check(L.pd_env_get_mass(self._h, _abi.dptr(self.mass), _abi.dptr(self.volume),
                                     _abi.dptr(self.density)))
        self.intact0 = np.zeros(self.N, dtype=np.int64)  # environment.jl:169
        _abi.check(L.pd_env_intact0(self._h, _abi.i64ptr(self.intact0)))
        y = self.y
        lo, hi = y.min(axis=1), y.max(axis=1)
        cm_, L_ = (lo + hi) / 2, hi - lo
        self.boundaries = (cm_ - (0.5 + self.bskin) * L_, cm_ + (0.5 + self.bskin) * L_)

    def _family(self, block):
        L = _abi.lib()
        rows = ctypes.c_int64()
        _abi.check(L.pd_env_family_rows(self._h, block, ctypes.byref(rows)))
        n = self.material_blocks[block].general.n
        fam = np.zeros((rows.value, n), dtype=np.int64, order="F")
        intact = np.zeros((rows.value, n), dtype=np.uint8, order="F")
        _abi.check(L.pd_env_get_family(self._h, block, _abi.i64ptr(fam), _abi.u8ptr(intact)))
        return fam, intact.astype(bool)

    def stage_state(self, slot):
        """Start an asynchronous snapshot of y, v, f and damage into staging
        slot 0 or 1 (the copy overlaps later steps)."""
        _abi.check(_abi.lib().pd_env_stage_state(self._h, int(slot)))

    def read_stage(self, slot):
        """Wait for a staged snapshot and return it (environment order)."""
        n = self.N
        y, v, f = (np.zeros((3, n), order="F") for _ in range(3))
        d = np.zeros(n)
        ts = ctypes.c_int64()
        _abi.check(_abi.lib().pd_env_stage_read(self._h, int(slot), _abi.dptr(y), _abi.dptr(v), _abi.dptr(f),
                                                _abi.dptr(d), ctypes.byref(ts)))
        return {"position": y, "velocity": v, "acceleration": f, "damage": d, "time_step": int(ts.value)}

    def _detach(self):
        """Give up ownership of the library handle (it now belongs to a
        server) and return it."""
        h, self._h = self._h, None
        return h

    def plastic_strain(self, block):
        """edp of an elasto-plastic block (rows x n, aligned with its family)."""
        L = _abi.lib()
        rows = ctypes.c_int64()
        _abi.check(L.pd_env_family_rows(self._h, block, ctypes.byref(rows)))
        n = self.material_blocks[block].general.n
        out = np.zeros((rows.value, n), order="F")
        _abi.check(L.pd_env_get_plastic_strain(self._h, block, _abi.dptr(out)))
        return out

    def kernel_shape(self):
        """(warps per slice, unroll) the throughput path runs with."""
        w, u = ctypes.c_int32(), ctypes.c_int32()
        _abi.check(_abi.lib().pd_env_kernel_shape(self._h, ctypes.byref(w), ctypes.byref(u)))
        return int(w.value), int(u.value)

    def set_kernel_shape(self, warps_per_slice=0, unroll=0):
        """Fix the throughput-mode kernel shape; (0, 0) = autotune."""
        _abi.check(_abi.lib().pd_env_set_kernel_shape(self._h, int(warps_per_slice), int(unroll)))

    def set_record_staging(self, mode=0):
        """FP32C record staging into shared memory: 0 = never (default),
        1 = staged shapes, 2 = the autotuner decides."""
        _abi.check(_abi.lib().pd_env_set_record_staging(self._h, int(mode)))

    def record_staging(self):
        """{'staged': running shape stages, 'slices': slices with a plan,
        'max_records': largest plan}."""
        st, sl, mx = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        _abi.check(_abi.lib().pd_env_record_staging(self._h, ctypes.byref(st), ctypes.byref(sl), ctypes.byref(mx)))
        return {"staged": bool(st.value), "slices": int(sl.value), "max_records": int(mx.value)}

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().pd_env_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_state(self):
        n = self.N
        y, v, f, p = (np.zeros((3, n), order="F") for _ in range(4))
        _abi.check(_abi.lib().pd_env_get_state(self._h, _abi.dptr(y), _abi.dptr(v), _abi.dptr(f), _abi.dptr(p)))
        return y, v, f, p

    def set_state(self, y=None, v=None, f=None):
        conv = (lambda a: None if a is None else np.asfortranarray(np.asarray(a, dtype=np.float64).reshape(3, -1)))
        y, v, f = conv(y), conv(v), conv(f)
        _abi.check(_abi.lib().pd_env_set_state(self._h, _abi.dptr(y), _abi.dptr(v), _abi.dptr(f)))

    def _get1(self, which):
        a = np.zeros((3, self.N), order="F")
        args = [None, None, None, None]
        args[which] = _abi.dptr(a)
        _abi.check(_abi.lib().pd_env_get_state(self._h, *args))
        return a

    y = property(lambda self: self._get1(0))
    v = property(lambda self: self._get1(1))
    f = property(lambda self: self._get1(2))
    p = property(lambda self: self._get1(3))

    @property
    def time_step(self):
        t = ctypes.c_int64()
        _abi.check(_abi.lib().pd_env_get_time_step(self._h, ctypes.byref(t)))
        return int(t.value)

    @time_step.setter
    def time_step(self, value):
        _abi.check(_abi.lib().pd_env_set_time_step(self._h, int(value)))

    def num_bonds(self):
        n = ctypes.c_int64()
        _abi.check(_abi.lib().pd_env_num_bonds(self._h, ctypes.byref(n)))
        return int(n.value)

    def contact_neighs(self, k):
        L = _abi.lib()
        rows = ctypes.c_int64()
        _abi.check(L.pd_env_get_contact_neighs(self._h, k, ctypes.byref(rows), None))
        cm = self.short_range_contact[k]
        n1 = cm.mat1.general.n
        out = np.zeros((rows.value, n1), dtype=np.int64, order="F")
        _abi.check(L.pd_env_get_contact_neighs(self._h, k, ctypes.byref(rows), _abi.i64ptr(out)))
        return out

    def theta(self, block):
        n = self.material_blocks[block].general.n
        t = np.zeros(n)
        _abi.check(_abi.lib().pd_env_get_theta(self._h, block, _abi.dptr(t)))
        return t

    def deformed(self):
        flags = np.zeros(len(self.material_blocks), dtype=np.uint8)
        _abi.check(_abi.lib().pd_env_deformed(self._h, _abi.u8ptr(flags)))
        return flags.astype(bool)

    def set_deformed(self, flags, hold=True):
        """Per-block deformed flags of the rigid-translation gate; with
        ``hold`` the library stops evaluating the gate itself."""
        f = np.ascontiguousarray(np.asarray(flags, dtype=np.uint8).reshape(-1))
        if f.size != len(self.material_blocks):
            raise ValueError("one flag per material block")
        _abi.check(_abi.lib().pd_env_set_deformed(self._h, _abi.u8ptr(f), int(bool(hold))))

    def layout(self):
        """Bond storage: slices, stencil slices, bond slots, index entries,
        slices with a record staging plan, slots the step kernels walk."""
        out = np.zeros(6, dtype=np.int64)
        _abi.check(_abi.lib().pd_env_layout_stats(self._h, _abi.i64ptr(out), 6))
        return {"slices": int(out[0]), "stencil_slices": int(out[1]), "slots": int(out[2]),
                "index_entries": int(out[3]), "staged_slices": int(out[4]), "walked_slots": int(out[5])}


def Env(id, materials, short_range_contact, boundary_conds, dt, state=2, bskin=0.5, units=False, **kwargs):
    """environment.jl:166-235 ``Env(id, materials, short_range_contact,
    boundary_conds, dt; state=2, bskin=0.5, units=false)``.  Extra keywords:
    ``precision`` ("fp64_serial", "fp64", "fp32c"), ``device``, ``families``
    (per block (family, intact) in the reference layout, or None)."""
    return GeneralEnvironment(id, materials, short_range_contact, boundary_conds, dt, state=state, bskin=bskin,
                              units=units, **kwargs)
