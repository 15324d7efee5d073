"""Slab decomposition host logic on the CPU: ownership, ghost layers deep
enough for complete families of owned and first-layer ghost particles,
the halo schedule, and the point-to-point exchange with two gloo ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import peridyn_b200 as pb
from peridyn_b200 import configs, lattice
from peridyn_b200.slabs import SlabPlan, SlabRank


def _bar():
    return configs.lps_bar(nx=40, ny=6, nz=5)


def _neighbours(x, h):
    d2 = ((x[:, :, None] - x[:, None, :]) ** 2).sum(axis=0)
    nb = (d2 < h * h)
    np.fill_diagonal(nb, False)
    return nb


@pytest.mark.parametrize("nslabs,axis", [(2, 0), (3, 0), (4, 0), (2, 1)])
def test_plan_ownership_and_ghost_depth(nslabs, axis):
    w = _bar()
    m = w["materials"][0]
    plan = SlabPlan(w["materials"], nslabs, axis=axis)
    n = m.general.n
    owned = np.zeros(n, dtype=np.int64)
    for s in range(nslabs):
        assert np.all(np.diff(plan.local[s]) > 0)  # environment order kept
        owned[plan.local[s][plan.owned[s]]] += 1
    assert np.all(owned == 1)
    nb = _neighbours(m.general.x, m.general.horizon)
    for s in range(nslabs):
        here = np.zeros(n, dtype=bool)
        here[plan.local[s]] = True
        own = plan.local[s][plan.owned[s]]
        first = np.unique(np.nonzero(nb[own])[1])
        assert here[first].all()  # owned families complete
        second = np.unique(np.nonzero(nb[first])[1])
        assert here[second].all()  # first-layer ghosts' families complete


@pytest.mark.parametrize("nslabs", [2, 3])
def test_plan_exchanges_cover_every_ghost_once(nslabs):
    w = _bar()
    plan = SlabPlan(w["materials"], nslabs)
    for s in range(nslabs):
        ghosts = plan.local[s][~plan.owned[s]]
        got = np.concatenate([plan.local[r][dst] for (o, r, src, dst) in plan.exchanges if r == s] or [[]])
        assert np.array_equal(np.sort(got.astype(np.int64)), np.sort(ghosts))
    for (o, s, src, dst) in plan.exchanges:
        assert np.array_equal(plan.local[o][src], plan.local[s][dst])
        assert np.all(plan.owner[plan.local[o][src]] == o)


def test_slab_workload_restricts_masks_and_keeps_types():
    x, vol = lattice.cuboid(20, 4, 4, 1e-3)
    t = np.where(x[0] < 10e-3, 1, 2).astype(np.int64)
    gen = pb.GeneralMaterial(x.copy(order="F"), np.zeros_like(x, order="F"), x, vol, t, 3.015e-3, max_neigh=200)
    mat = pb.PeridynamicsMaterial(gen, pb.BondBasedSpecific([10e9, 11e9, 12e9], [0.01, 0.01, 0.01], [2000.0, 2100.0]))
    bcs = [pb.FixBC(x[0] < 2e-3)]
    plan = SlabPlan([mat], 2)
    for s in range(2):
        mats, sbcs = plan.slab_workload(s, [mat], bcs)
        assert mats[0].type == mat.type
        assert np.array_equal(sbcs[0].bool, bcs[0].bool[plan.local[s]])
        assert mats[0].general.particle_size == gen.particle_size


class _FakeSlab:
    """State rows (9 values per local particle) standing for a slab's
    environment: pack/unpack move rows by local index."""

    def __init__(self, rows):
        self.rows = rows

    def pack(self, idx, buf):
        buf.view(-1, 9)[:] = self.rows[idx]

    def unpack(self, idx, buf):
        self.rows[idx] = buf.view(-1, 9)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, nslabs, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = _bar()
        plan = SlabPlan(w["materials"], nslabs)
        loc = plan.local[rank]
        rows = torch.zeros((loc.size, 9), dtype=torch.float64)
        own = torch.as_tensor(plan.owned[rank])
        # owned rows carry their global index; ghost rows start at -1
        rows[own] = torch.as_tensor(loc[plan.owned[rank]], dtype=torch.float64)[:, None] + torch.arange(9) / 10
        rows[~own] = -1.0
        SlabRank(plan, rank, dist, _FakeSlab(rows), device="cpu").exchange()
        expect = torch.as_tensor(loc, dtype=torch.float64)[:, None] + torch.arange(9) / 10
        out[rank] = bool(torch.equal(rows, expect))
    finally:
        dist.destroy_process_group()


class _FakeDiag:
    """Per-particle values standing for a slab's state: owned_sums returns
    the local sums SlabRank.diagnostics reduces."""

    def __init__(self, vals):
        self.vals = vals  # (n, 9): p (3), f (3), damage, 1, intact bonds

    def owned_sums(self, own):
        return self.vals[own].sum(axis=0)


def _diag_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = _bar()
        plan = SlabPlan(w["materials"], world)
        loc = plan.local[rank]
        g = loc.astype(np.float64)  # values keyed by the global index: ghosts repeat owners' rows
        vals = np.stack([g, 2 * g, -g, g, 0 * g, 1 + 0 * g, 0.5 + 0 * g, 1 + 0 * g, 10 + 0 * g], axis=1)
        d = SlabRank(plan, rank, dist, _FakeDiag(vals), device="cpu").diagnostics()
        out[rank] = (list(d["p"]), list(d["f"]), d["damage"], d["bonds"])
    finally:
        dist.destroy_process_group()


def test_two_rank_diagnostics_allreduce_gloo():
    """The body's sums counted once: owned particles only, summed over the
    ranks; every rank gets the same totals."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_diag_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    n = _bar()["materials"][0].general.n
    s = n * (n - 1) / 2
    assert out[0] == out[1]
    p, f, dmg, bonds = out[0]
    assert p == [s, 2 * s, -s] and f == [s, 0.0, float(n)]
    assert dmg == 0.5 and bonds == 10 * n


def test_two_rank_halo_exchange_gloo():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, 2, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] and out[1]


def test_rank_wire_must_be_device_or_host():
    w = _bar()
    plan = SlabPlan(w["materials"], 2)
    with pytest.raises(ValueError):
        SlabRank(plan, 0, dist, _FakeSlab(torch.zeros((plan.local[0].size, 9))), device="cpu", wire="nvlink")


def _disk_with_contact():
    return configs.disk_impact(radius=3.0e-3, thickness=1.0e-3, spacing=2.5e-4, sphere_radius=1.0e-3, speed=100.0)


@pytest.mark.parametrize("nslabs,axis", [(2, 0), (3, 0), (2, 1)])
def test_plan_contact_partners_and_their_candidates_are_local(nslabs, axis):
    """Two-block contact in slabs: for every owned particle of either block,
    its contact partners (other block, within the search distance) and
    their own candidates are in the slab, so the slab's contact lists and
    reactions are the whole body's."""
    w = _disk_with_contact()
    cm = w["contacts"][0]
    m1, m2 = w["materials"]
    plan = SlabPlan(w["materials"], nslabs, axis=axis, contacts=w["contacts"])
    x = np.hstack([m1.general.x, m2.general.x])
    n1 = m1.general.n
    d2 = ((x[:, :n1, None] - x[:, None, n1:]) ** 2).sum(axis=0)
    near = d2 < cm.distance ** 2  # n1 x n2 candidate pairs
    for s in range(nslabs):
        here = np.zeros(x.shape[1], dtype=bool)
        here[plan.local[s]] = True
        own = plan.local[s][plan.owned[s]]
        own1, own2 = own[own < n1], own[own >= n1] - n1
        p2 = np.unique(np.nonzero(near[own1])[1])  # partners of owned block-1 particles
        p1 = np.unique(np.nonzero(near[:, own2])[0])  # partners of owned block-2 particles
        assert here[n1 + p2].all() and here[p1].all()
        assert here[np.unique(np.nonzero(near[:, p2])[0])].all()  # candidates of those partners
        assert here[n1 + np.unique(np.nonzero(near[p1])[1])].all()
    mats, _, scs = plan.slab_workload(0, w["materials"], [], w["contacts"])
    assert len(scs) == 1 and scs[0].mat1 is mats[0] and scs[0].mat2 is mats[1]


def test_plan_rejects_self_contact():
    x, vol = lattice.cuboid(8, 4, 4, 1e-3)
    gen = pb.GeneralMaterial(x.copy(order="F"), np.zeros_like(x, order="F"), x, vol, np.ones(x.shape[1], np.int64),
                             3.015e-3, max_neigh=200)
    mat = pb.PeridynamicsMaterial(gen, pb.BondBasedSpecific([10e9], [0.01], [2000.0]))
    with pytest.raises(TypeError):
        SlabPlan([mat], 2, contacts=[pb.LinearSpringContactModel(1e18, mat)])
