"""Slab decomposition with one process per slab (``SlabRank``): two ranks,
each holding its slab environment on the GPU, exchange halos through
``torch.distributed`` point-to-point (gloo, host-staged buffers) after
every velocity-Verlet step.  The owned particles' states must equal the
whole body run as one environment: bit for bit in the serial FP64 mode,
within 1e-4 relative-L2 of the displacement in FP32C.

The ranks share one GPU but never wait on each other inside a kernel:
every exchange completes on the host between steps."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _workload():
    from peridyn_b200 import configs

    return configs.lps_bar(nx=48, ny=8, nz=8, steps=40)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, precision, nsteps, out):
    import torch.distributed as dist

    import peridyn_b200 as pb
    from peridyn_b200.slabs import SlabPlan, SlabRank

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = _workload()
        plan = SlabPlan(w["materials"], world)
        mats, bcs = plan.slab_workload(rank, w["materials"], w["bcs"])
        env = pb.Env(1, mats, [], bcs, w["dt"], precision=precision, device=0)
        env.set_deformed(np.ones(len(mats), dtype=np.uint8), hold=True)
        pb.apply_bc_at0(env, 0)
        r = SlabRank(plan, rank, dist, env, device="cuda:0", wire="host")
        r.step(nsteps)
        out[rank] = r.owned_state()
        out[f"diag{rank}"] = r.diagnostics()
        env.close()
    finally:
        dist.destroy_process_group()


def _whole(w, precision, nsteps):
    import peridyn_b200 as pb

    env = pb.Env(1, w["materials"], [], w["bcs"], w["dt"], precision=precision)
    env.set_deformed(np.ones(len(w["materials"]), dtype=np.uint8), hold=True)
    pb.apply_bc_at0(env, 0)
    pb.velocity_verlet_step(env, nsteps=nsteps)
    y, v, f, pm = env.get_state()
    diag = np.zeros(8)
    from peridyn_b200 import _abi

    _abi.check(_abi.lib().pd_env_diagnostics(env._h, _abi.dptr(diag)))
    env.close()
    return y, v, f, diag, pm


@pytest.mark.parametrize("precision", ["fp64_serial", "fp32c"])
def test_two_slab_ranks_match_whole_body(precision):
    nsteps = 40
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, precision, nsteps, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.exitcode is None:
            p.kill()
        assert p.exitcode == 0

    w = _workload()
    y0, v0, f0, diag, p0 = _whole(w, precision, nsteps)
    n = y0.shape[1]
    y1, v1, f1 = np.full((3, n), np.nan), np.full((3, n), np.nan), np.full((3, n), np.nan)
    for rank in range(2):
        idx, ys, vs, fs = out[rank]
        y1[:, idx], v1[:, idx], f1[:, idx] = ys, vs, fs
    assert not np.isnan(y1).any()  # every particle owned by exactly one rank
    # the ranks' all-reduced diagnostics: the whole body's, counted once
    d0, d1 = out["diag0"], out["diag1"]
    assert np.array_equal(d0["p"], d1["p"]) and d0["bonds"] == d1["bonds"]
    assert d0["bonds"] == int(diag[7])
    # the sums nearly cancel, so they are compared on the scale of their
    # summands: the force sum against the ranks' own owned forces (round-off
    # of the summation order), the momentum against the whole body's (equal
    # states in serial FP64, within the FP32C state tolerance otherwise)
    tol_p = 1e-12 if precision == "fp64_serial" else 1e-4
    for got, ref, parts, tol in ((d0["p"], diag[0:3], p0, tol_p), (d0["f"], f1.sum(axis=1), f1, 1e-12)):
        scale = np.abs(parts).sum(axis=1) + 1e-300
        assert np.all(np.abs(np.asarray(got) - ref) <= tol * scale), (got, ref, scale)
    if precision == "fp64_serial":
        assert np.all(np.abs(np.asarray(d0["f"]) - diag[3:6]) <= 1e-12 * np.abs(f0).sum(axis=1))
    assert abs(d0["damage"] - diag[6]) <= 1e-12
    if precision == "fp64_serial":
        assert np.array_equal(y0, y1)
        assert np.array_equal(v0, v1)
        assert np.array_equal(f0, f1)
    else:
        x = w["materials"][0].general.x
        du = np.linalg.norm((y1 - x) - (y0 - x)) / np.linalg.norm(y0 - x)
        assert du <= 1e-4, du
