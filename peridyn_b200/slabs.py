"""Slab decomposition of one specimen (the multi-GPU plan for a single
large body; the reference runs one body on one device).

The body is cut along one axis into slabs of equal particle count.  Each
slab is an environment of its own: the particles it owns plus ghost
layers on either side, taken from the reference configuration, in the
same relative (environment) order as in the whole body.  The ghost depth
is what the owned particles' terms reach: two horizons for bond-based and
state-based blocks (an owned particle reads the dilatation of its
neighbours, which needs their complete families), three with
elasto-plastic blocks (a yielding neighbour's td_norm2 reads the
dilatation of its own neighbours).  An owned particle then sees exactly
the neighbours, weighted volumes, dilatations, plastic history and bond
flags it has in the whole body.
After every velocity-Verlet step the owners' state (q, v, f; see
``pd_env_pack_halo``) is copied into the ghosts that stand for them, the
one halo exchange per step.  Ghosts are integrated by their slab as well,
but their results are replaced by the owners' before they are read.

The rigid-translation gate (general_material.jl:240-256) is a property of
a whole block: decided on one slab's particles it would switch at other
steps (its tolerance is relative to the particles it sees).  Slabs
therefore hold every block deformed from the first step
(``pd_env_set_deformed``), as a whole-body run with the gate held open
does; forces skipped by the gate are those of a rigid translation.

In the serial FP64 mode the slabs reproduce such a whole-body run bit for
bit (the gather order per particle follows the global indices, which the
slabs keep); the throughput modes sum each particle's bonds over a
different slice layout, within their stated tolerances.  Contact models
are not supported in slab mode.

``SlabRun`` runs all slabs in one process (one device, or one device per
slab); ``SlabRank`` is one slab per ``torch.distributed`` rank, the halo
buffers moving by point-to-point send/recv (NCCL between GPUs).  The
exchange schedule (``SlabPlan.exchanges``) is the same for both.
"""
import copy

import numpy as np

from . import _abi
from .environment import Env
from .materials import GeneralMaterial, PeridynamicsMaterial


class SlabPlan:
    """Ownership, ghosts and the halo schedule of ``nslabs`` slabs along
    ``axis`` for the given material blocks (environment order = blocks in
    order).  ``halo`` is the ghost depth in horizons; None: 3 with
    elasto-plastic blocks, else 2."""

    def __init__(self, materials, nslabs, axis=0, halo=None):
        if nslabs < 1:
            raise ValueError("nslabs must be >= 1")
        if halo is None:
            halo = 3.0 if any(m.kind == _abi.PD_MAT_ELASTO_PLASTIC for m in materials) else 2.0
        self.halo = float(halo)
        self.nslabs = int(nslabs)
        self.axis = int(axis)
        xs, blk, hor = [], [], []
        for b, m in enumerate(materials):
            g = m.general
            xs.append(g.x)
            blk.append(np.full(g.n, b, dtype=np.int64))
            hor.append(np.full(g.n, g.horizon))
        x = np.hstack(xs)
        self.block = np.concatenate(blk)
        self.n = x.shape[1]
        c = x[self.axis]
        # cuts at particle-count quantiles of the axis coordinate
        order = np.argsort(c, kind="stable")
        owner = np.empty(self.n, dtype=np.int64)
        bounds = np.linspace(0, self.n, self.nslabs + 1).round().astype(np.int64)
        for s in range(self.nslabs):
            owner[order[bounds[s]:bounds[s + 1]]] = s
        self.owner = owner
        reach = halo * np.concatenate(hor) * (1.0 + 1e-9)
        self.local = []  # per slab: environment-order indices of its particles, ascending
        self.owned = []  # per slab: bool over its local particles
        for s in range(self.nslabs):
            mine = owner == s
            if not mine.any():
                raise ValueError(f"slab {s} owns no particle")
            lo, hi = c[mine].min(), c[mine].max()
            near = (c >= lo - reach) & (c <= hi + reach)
            sel = np.nonzero(mine | near)[0]
            self.local.append(sel)
            self.owned.append(mine[sel])
        # exchanges: (owner slab, receiving slab, owner-local idx, receiver-local idx)
        self.exchanges = []
        for s in range(self.nslabs):
            ghosts = self.local[s][~self.owned[s]]
            for o in range(self.nslabs):
                if o == s:
                    continue
                g = ghosts[owner[ghosts] == o]
                if g.size == 0:
                    continue
                src = np.searchsorted(self.local[o], g)
                dst = np.searchsorted(self.local[s], g)
                self.exchanges.append((o, s, src.astype(np.int64), dst.astype(np.int64)))

    def slab_workload(self, s, materials, bcs):
        """Materials and BCs of slab s: per block its particles (owned and
        ghost) with the block's parameters; BC masks restricted to them."""
        sel = self.local[s]
        mats = []
        for b, m in enumerate(materials):
            first = int(np.sum(self.block < b))
            pick = sel[self.block[sel] == b] - first
            if pick.size == 0:
                continue
            g = m.general
            sub = GeneralMaterial(g.y[:, pick], g.velocity[:, pick], g.x[:, pick], g.volume[pick], g.type[pick],
                                  g.horizon, max_neigh=g.max_neigh, particle_size=g.particle_size,
                                  skip_bb=g.skip_bb)
            pm = PeridynamicsMaterial(sub, copy.copy(m.specific), name=f"{m.name}[slab {s}]")
            pm.type = m.type  # the block's type range, whether or not all types occur here
            mats.append(pm)
        sub_bcs = []
        for bc in bcs:
            c = copy.copy(bc)
            c.bool = np.ascontiguousarray(np.asarray(bc.bool, dtype=np.uint8)[sel])
            sb = getattr(bc, "scalebool", None)
            if sb is not None:
                c.scalebool = np.ascontiguousarray(np.asarray(sb, dtype=np.uint8)[sel])
            sub_bcs.append(c)
        return mats, sub_bcs


def _torch():
    import torch

    return torch


class SlabRun:
    """All slabs of one body in one process.  ``devices``: one CUDA device
    index per slab (default: all on device 0).  ``step(n)`` advances every
    slab n velocity-Verlet steps with a halo exchange after each;
    ``state()`` gathers y, v, f of the owned particles in environment
    order."""

    def __init__(self, materials, bcs, dt, nslabs, axis=0, precision="fp64_serial", devices=None, halo=None):
        if any(getattr(m, "kind", None) is None for m in materials):
            raise TypeError("materials must be PeridynamicsMaterial blocks")
        self.plan = SlabPlan(materials, nslabs, axis=axis, halo=halo)
        self.devices = list(devices) if devices is not None else [0] * nslabs
        self.envs = []
        for s in range(nslabs):
            mats, sbcs = self.plan.slab_workload(s, materials, bcs)
            env = Env(1, mats, [], sbcs, dt, precision=precision, device=self.devices[s])
            env.set_deformed(np.ones(len(mats), dtype=np.uint8), hold=True)
            self.envs.append(env)
        torch = _torch()
        self._idx = []
        for (o, s, src, dst) in self.plan.exchanges:
            self._idx.append((torch.as_tensor(src, device=f"cuda:{self.devices[o]}"),
                              torch.as_tensor(dst, device=f"cuda:{self.devices[s]}"),
                              torch.empty(9 * src.size, dtype=torch.float64, device=f"cuda:{self.devices[o]}")))

    def apply_bc_at0(self):
        for e in self.envs:
            _abi.check(_abi.lib().pd_env_apply_bc_at0(e._h))

    def _sync(self):
        torch = _torch()
        for d in sorted(set(self.devices)):
            torch.cuda.synchronize(d)

    def exchange(self):
        """Owners' (q, v, f) into the ghosts standing for them."""
        L = _abi.lib()
        self._sync()
        for (o, s, _, _), (src, _, buf) in zip(self.plan.exchanges, self._idx):
            _abi.check(L.pd_env_pack_halo(self.envs[o]._h, src.data_ptr(), src.numel(), buf.data_ptr()))
        self._sync()
        # copies between devices run on torch's streams: complete them before
        # the environments' streams unpack
        bufs = [buf if self.devices[o] == self.devices[s] else buf.to(f"cuda:{self.devices[s]}")
                for (o, s, _, _), (_, _, buf) in zip(self.plan.exchanges, self._idx)]
        self._sync()
        for (o, s, _, _), (_, dst, _), b in zip(self.plan.exchanges, self._idx, bufs):
            _abi.check(L.pd_env_unpack_halo(self.envs[s]._h, dst.data_ptr(), dst.numel(), b.data_ptr()))
        self._sync()

    def step(self, nsteps=1):
        L = _abi.lib()
        for _ in range(int(nsteps)):
            for e in self.envs:
                _abi.check(L.pd_env_vv_steps(e._h, 1))
            self.exchange()

    def state(self):
        n = self.plan.n
        y, v, f = np.zeros((3, n), order="F"), np.zeros((3, n), order="F"), np.zeros((3, n), order="F")
        for s, e in enumerate(self.envs):
            ys, vs, fs, _ = e.get_state()
            own = self.plan.owned[s]
            idx = self.plan.local[s][own]
            y[:, idx], v[:, idx], f[:, idx] = ys[:, own], vs[:, own], fs[:, own]
        return y, v, f

    def close(self):
        for e in self.envs:
            e.close()
        self.envs = []


class SlabRank:
    """One slab per ``torch.distributed`` rank (world size = number of
    slabs): the halo buffers of the plan's exchanges move by point-to-point
    send/recv, each rank sending what it owns and receiving its ghosts, in
    the plan's order on every rank.  ``env`` is the rank's slab
    environment (an ``Env`` built from ``plan.slab_workload(rank, ...)`` on
    the rank's device) or any object with ``pack(idx, buf)`` /
    ``unpack(idx, buf)`` on tensors.  ``wire`` is where the send/recv
    buffers live: ``"device"`` (NCCL moves device memory) or ``"host"``
    (pinned host copies, for a backend without device tensors such as
    gloo)."""

    def __init__(self, plan, rank, dist, env, device="cuda", wire="device"):
        if wire not in ("device", "host"):
            raise ValueError("wire must be 'device' or 'host'")
        self.plan, self.rank, self.dist, self.device = plan, int(rank), dist, device
        self.env = env
        torch = _torch()
        on_dev = str(device).startswith("cuda")
        self.host_wire = wire == "host" and on_dev

        def wire_buf(n):
            if self.host_wire:
                return torch.empty(9 * n, dtype=torch.float64, pin_memory=True)
            return None

        self.sends, self.recvs = [], []
        for (o, s, src, dst) in plan.exchanges:
            if o == self.rank:
                self.sends.append((s, torch.as_tensor(src, device=device),
                                   torch.empty(9 * src.size, dtype=torch.float64, device=device),
                                   wire_buf(src.size)))
            if s == self.rank:
                self.recvs.append((o, torch.as_tensor(dst, device=device),
                                   torch.empty(9 * dst.size, dtype=torch.float64, device=device),
                                   wire_buf(dst.size)))

    def _pack(self, idx, buf):
        if hasattr(self.env, "pack"):
            self.env.pack(idx, buf)
        else:
            _abi.check(_abi.lib().pd_env_pack_halo(self.env._h, idx.data_ptr(), idx.numel(), buf.data_ptr()))

    def _unpack(self, idx, buf):
        if hasattr(self.env, "unpack"):
            self.env.unpack(idx, buf)
        else:
            _abi.check(_abi.lib().pd_env_unpack_halo(self.env._h, idx.data_ptr(), idx.numel(), buf.data_ptr()))

    def _sync(self):
        # the environment's stream (pack/unpack) and torch's stream (copies,
        # NCCL) are not ordered with each other: wait for the whole device
        if str(self.device).startswith("cuda"):
            _torch().cuda.synchronize(self.device)

    def exchange(self):
        for _, idx, buf, _ in self.sends:
            self._pack(idx, buf)
        self._sync()
        if self.host_wire:
            for _, _, buf, hbuf in self.sends:
                hbuf.copy_(buf)
        ops = [self.dist.P2POp(self.dist.isend, buf if hbuf is None else hbuf, peer)
               for peer, _, buf, hbuf in self.sends]
        ops += [self.dist.P2POp(self.dist.irecv, buf if hbuf is None else hbuf, peer)
                for peer, _, buf, hbuf in self.recvs]
        if ops:
            for r in self.dist.batch_isend_irecv(ops):
                r.wait()
        if self.host_wire:
            for _, _, buf, hbuf in self.recvs:
                buf.copy_(hbuf)
        self._sync()  # received (or copied) halo data complete before the unpack reads it
        for _, idx, buf, _ in self.recvs:
            self._unpack(idx, buf)

    def step(self, nsteps=1):
        """``nsteps`` velocity-Verlet steps of the rank's slab, a halo
        exchange after each (every rank calls it with the same count)."""
        L = _abi.lib()
        for _ in range(int(nsteps)):
            _abi.check(L.pd_env_vv_steps(self.env._h, 1))
            self.exchange()

    def owned_state(self):
        """(environment-order indices, y, v, f) of the particles this rank
        owns."""
        ys, vs, fs, _ = self.env.get_state()
        own = self.plan.owned[self.rank]
        return self.plan.local[self.rank][own], ys[:, own], vs[:, own], fs[:, own]
