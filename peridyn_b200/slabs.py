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
different slice layout, within their stated tolerances.

Two-block contact (ContactModel12, contacts.jl:189-247 and 434-476) runs
in every slab holding particles of both blocks, between the slab's parts
of them.  The ghost layers are then at least twice the contact search
distance deep as well: a contact partner of an owned particle lies within
one search distance, and that partner's own candidates (whose top
max_neighs by index the search keeps) within two, so both lists come out
as in the whole body, and the slab's relative order keeps the selection
and the force gather order.  Each slab rebuilds its contact lists itself
(``update_neighs``).  Self contact (ContactModel11) reads bond flags of
ghost particles, which the halo exchange does not carry; it is rejected.

``SlabRun`` runs all slabs in one process (one device, or one device per
slab); ``SlabRank`` is one slab per ``torch.distributed`` rank, the halo
buffers moving by point-to-point send/recv (NCCL between GPUs).  The
exchange schedule (``SlabPlan.exchanges``) is the same for both.
"""
import copy
import ctypes

import numpy as np

from . import _abi
from .contacts import NonLinearSpringContactModel12
from .environment import Env
from .materials import GeneralMaterial, PeridynamicsMaterial


class SlabPlan:
    """Ownership, ghosts and the halo schedule of ``nslabs`` slabs along
    ``axis`` for the given material blocks (environment order = blocks in
    order).  ``halo`` is the ghost depth in horizons; None: 3 with
    elasto-plastic blocks, else 2."""

    def __init__(self, materials, nslabs, axis=0, halo=None, contacts=()):
        if nslabs < 1:
            raise ValueError("nslabs must be >= 1")
        for cm in contacts:
            if not isinstance(cm, NonLinearSpringContactModel12):
                raise TypeError("slab mode supports two-block contact models only (self contact reads ghost "
                                "bond flags, which the halo exchange does not carry)")
        if halo is None:
            halo = 3.0 if any(m.kind == _abi.PD_MAT_ELASTO_PLASTIC for m in materials) else 2.0
        self.halo = float(halo)
        # contact partners and their candidates: two search distances
        self.contact_reach = 2.0 * max([cm.distance for cm in contacts], default=0.0)
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
        reach = np.maximum(halo * np.concatenate(hor), self.contact_reach) * (1.0 + 1e-9)
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

    def slab_workload(self, s, materials, bcs, contacts=()):
        """Materials, BCs and contact models of slab s: per block its
        particles (owned and ghost) with the block's parameters; BC masks
        restricted to them; each two-block contact model between the slab's
        parts of its blocks (dropped where the slab lacks one of them).
        With ``contacts`` given, returns (materials, bcs, contacts)."""
        sel = self.local[s]
        mats = []
        sub_of = {}
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
            sub_of[id(m)] = pm
        sub_bcs = []
        for bc in bcs:
            c = copy.copy(bc)
            c.bool = np.ascontiguousarray(np.asarray(bc.bool, dtype=np.uint8)[sel])
            sb = getattr(bc, "scalebool", None)
            if sb is not None:
                c.scalebool = np.ascontiguousarray(np.asarray(sb, dtype=np.uint8)[sel])
            sub_bcs.append(c)
        if not contacts:
            return mats, sub_bcs
        sub_contacts = []
        for cm in contacts:
            m1, m2 = sub_of.get(id(cm.mat1)), sub_of.get(id(cm.mat2))
            if m1 is None or m2 is None:
                continue
            c = copy.copy(cm)
            c.mat1, c.mat2 = m1, m2
            c.max_neighs = min(cm.max_neighs, m2.general.n)
            sub_contacts.append(c)
        return mats, sub_bcs, sub_contacts


def _torch():
    import torch

    return torch


def env_stream(env, device):
    """The environment's CUDA stream as a torch stream (for event ordering)."""
    torch = _torch()
    sp = ctypes.c_void_p()
    _abi.check(_abi.lib().pd_env_stream(env._h, ctypes.byref(sp)))
    return torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", device))


class SlabRun:
    """All slabs of one body in one process.  ``devices``: one CUDA device
    index per slab (default: all on device 0).  ``step(n)`` advances every
    slab n velocity-Verlet steps with a halo exchange after each;
    ``state()`` gathers y, v, f of the owned particles in environment
    order."""

    def __init__(self, materials, bcs, dt, nslabs, axis=0, precision="fp64_serial", devices=None, halo=None,
                 contacts=()):
        if any(getattr(m, "kind", None) is None for m in materials):
            raise TypeError("materials must be PeridynamicsMaterial blocks")
        self.plan = SlabPlan(materials, nslabs, axis=axis, halo=halo, contacts=contacts)
        self.devices = list(devices) if devices is not None else [0] * nslabs
        self.envs = []
        for s in range(nslabs):
            if contacts:
                mats, sbcs, scs = self.plan.slab_workload(s, materials, bcs, contacts)
            else:
                (mats, sbcs), scs = self.plan.slab_workload(s, materials, bcs), []
            env = Env(1, mats, scs, sbcs, dt, precision=precision, device=self.devices[s])
            env.set_deformed(np.ones(len(mats), dtype=np.uint8), hold=True)
            self.envs.append(env)
        torch = _torch()
        self._idx = []
        for (o, s, src, dst) in self.plan.exchanges:
            cross = self.devices[o] != self.devices[s]
            self._idx.append((torch.as_tensor(src, device=f"cuda:{self.devices[o]}"),
                              torch.as_tensor(dst, device=f"cuda:{self.devices[s]}"),
                              torch.empty(9 * src.size, dtype=torch.float64, device=f"cuda:{self.devices[o]}"),
                              torch.empty(9 * src.size, dtype=torch.float64, device=f"cuda:{self.devices[s]}")
                              if cross else None))
        self._streams = [env_stream(e, d) for e, d in zip(self.envs, self.devices)]
        self._copy = {d: torch.cuda.Stream(device=d) for d in set(self.devices)}
        # per exchange: the event after which its send buffer / receive
        # buffer may be overwritten (the last reader has finished)
        self._free_send = [None] * len(self.plan.exchanges)
        self._free_recv = [None] * len(self.plan.exchanges)

    def apply_bc_at0(self):
        for e in self.envs:
            _abi.check(_abi.lib().pd_env_apply_bc_at0(e._h))

    def update_neighs(self, max_part=30):
        """update_neighs! (solvers.jl:351-361) in every slab."""
        for e in self.envs:
            _abi.check(_abi.lib().pd_env_update_neighs(e._h, int(max_part)))

    def update_acc(self):
        """update_acc! in every slab (forces at the current positions, e.g.
        save_state! at t0); ghosts receive their owners' values."""
        for e in self.envs:
            _abi.check(_abi.lib().pd_env_update_acc(e._h))
        self.exchange()

    def _sync(self):
        torch = _torch()
        for d in sorted(set(self.devices)):
            torch.cuda.synchronize(d)

    def exchange(self):
        """Owners' (q, v, f) into the ghosts standing for them, ordered on
        the device by CUDA events, without host waits: pack on the owner's
        stream, the copy between GPUs on a copy stream of the receiving GPU,
        unpack on the receiver's stream, and the next pack into a buffer
        only after its last reader."""
        torch = _torch()
        L = _abi.lib()
        for k, ((o, s, _, _), (src, dst, buf, rbuf)) in enumerate(zip(self.plan.exchanges, self._idx)):
            so, ss = self._streams[o], self._streams[s]
            if self._free_send[k] is not None:
                so.wait_event(self._free_send[k])
            _abi.check(L.pd_env_pack_halo(self.envs[o]._h, src.data_ptr(), src.numel(), buf.data_ptr()))
            packed = torch.cuda.Event()
            packed.record(so)
            if rbuf is None:
                ss.wait_event(packed)
                src_buf = buf
            else:
                cs = self._copy[self.devices[s]]
                cs.wait_event(packed)
                if self._free_recv[k] is not None:
                    cs.wait_event(self._free_recv[k])
                with torch.cuda.stream(cs):
                    rbuf.copy_(buf, non_blocking=True)
                moved = torch.cuda.Event()
                moved.record(cs)
                self._free_send[k] = moved
                ss.wait_event(moved)
                src_buf = rbuf
            _abi.check(L.pd_env_unpack_halo(self.envs[s]._h, dst.data_ptr(), dst.numel(), src_buf.data_ptr()))
            unpacked = torch.cuda.Event()
            unpacked.record(ss)
            if rbuf is None:
                self._free_send[k] = unpacked
            else:
                self._free_recv[k] = unpacked

    def step(self, nsteps=1):
        """nsteps velocity-Verlet steps of every slab, a halo exchange
        after each; the slabs' steps are enqueued without host waits
        (pd_env_vv_steps_async: their gates are held), so slabs on
        different GPUs run at once.  Returns when all have finished."""
        L = _abi.lib()
        for _ in range(int(nsteps)):
            for e in self.envs:
                _abi.check(L.pd_env_vv_steps_async(e._h, 1))
            self.exchange()
        self._sync()

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

        # the slab environment's stream, for event ordering on the device wire
        self._env_stream = env_stream(env, torch.device(device).index or 0) \
            if (on_dev and hasattr(env, "_h")) else None
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
        torch = _torch()
        for _, idx, buf, _ in self.sends:
            self._pack(idx, buf)
        if not self.host_wire and self._env_stream is not None:
            # device wire: NCCL runs on torch's current stream; order it after
            # the packs, and the unpacks after it, with events (no host wait)
            packed = torch.cuda.Event()
            packed.record(self._env_stream)
            torch.cuda.current_stream(self.device).wait_event(packed)
            ops = [self.dist.P2POp(self.dist.isend, buf, peer) for peer, _, buf, _ in self.sends]
            ops += [self.dist.P2POp(self.dist.irecv, buf, peer) for peer, _, buf, _ in self.recvs]
            if ops:
                for r in self.dist.batch_isend_irecv(ops):
                    r.wait()
            done = torch.cuda.Event()
            done.record(torch.cuda.current_stream(self.device))
            self._env_stream.wait_event(done)
            for _, idx, buf, _ in self.recvs:
                self._unpack(idx, buf)
            return
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
        run = L.pd_env_vv_steps_async if self._env_stream is not None and not self.host_wire else L.pd_env_vv_steps
        for _ in range(int(nsteps)):
            _abi.check(run(self.env._h, 1))
            self.exchange()
        if self._env_stream is not None:
            self._env_stream.synchronize()

    def diagnostics(self):
        """printdata's sums (environment.jl:308-320) over the whole body:
        momentum and force sums, mean damage and intact bonds of the
        particles each rank owns (ghosts excluded), summed over the ranks
        by one all-reduce (NCCL on the device wire, else on the host).
        Returns {"p": (3,), "f": (3,), "damage": mean, "bonds": count}."""
        torch = _torch()
        own = np.asarray(self.plan.owned[self.rank])
        if hasattr(self.env, "owned_sums"):
            local = np.asarray(self.env.owned_sums(own), dtype=np.float64)
        else:
            _, _, f, p = self.env.get_state()
            d = np.zeros(own.size)
            _abi.check(_abi.lib().pd_env_damage(self.env._h, _abi.dptr(d)))
            i0 = np.asarray(self.env.intact0, dtype=np.float64)
            local = np.concatenate([p[:, own].sum(axis=1), f[:, own].sum(axis=1),
                                    [d[own].sum(), float(own.sum()), ((1.0 - d[own]) * i0[own]).sum()]])
        dev = self.device if (str(self.device).startswith("cuda") and not self.host_wire) else "cpu"
        t = torch.as_tensor(local, dtype=torch.float64, device=dev)
        self.dist.all_reduce(t)
        g = t.cpu().numpy()
        return {"p": g[0:3], "f": g[3:6], "damage": g[6] / max(g[7], 1.0), "bonds": int(round(g[8]))}

    def owned_state(self):
        """(environment-order indices, y, v, f) of the particles this rank
        owns."""
        ys, vs, fs, _ = self.env.get_state()
        own = self.plan.owned[self.rank]
        return self.plan.local[self.rank][own], ys[:, own], vs[:, own], fs[:, own]
