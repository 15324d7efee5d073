"""Serving loop (pd_server_*): continuous batching on one GPU.  A job's
result is the same alone and in a mix (bit-identical: each job runs its own
kernels with a shape fixed from its size), and equals a direct run of the
same simulation through Env."""
import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import _abi, configs

pytestmark = pytest.mark.gpu


def _jobs():
    a = configs.pmb_cube(dims=(12, 11, 10), peak=40.0, cs=0.003, steps=150)
    b = configs.lps_cube((10, 9, 9), peak=30.0, steps=200)
    c = configs.pmb_cube(dims=(16, 14, 12), peak=20.0, seed=3, steps=120)
    d = configs.lps_bar(nx=30, ny=8, nz=8, steps=180)  # Fix + Move BCs
    return [a, b, c, d]


def _submit(srv, w, precision):
    return srv.submit(w["materials"], w["contacts"], w["bcs"], w["dt"], w["steps"], precision=precision)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_same_result_alone_and_in_mix(precision):
    jobs = _jobs()
    alone = []
    with pb.Server(max_active=1) as srv:
        for w in jobs:
            j = _submit(srv, w, precision)
            info = srv.wait(j)
            assert info["state"] == "done" and info["steps_done"] == w["steps"]
            alone.append(srv.result(j))
    with pb.Server(max_active=8, chunk_steps=64) as srv:
        ids = [_submit(srv, w, precision) for w in jobs]
        infos = [srv.wait(j) for j in ids]
        mixed = [srv.result(j) for j in ids]
    assert all(i["state"] == "done" for i in infos)
    for r1, r2 in zip(alone, mixed):
        for a, b in zip(r1, r2):
            assert np.array_equal(a, b)


def test_server_matches_direct_run():
    w = configs.lps_bar(nx=30, ny=8, nz=8, steps=180)
    with pb.Server() as srv:
        j = _submit(srv, w, "fp32c")
        srv.wait(j)
        y, v, d = srv.result(j)
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision="fp32c")
    slices = env.layout()["slices"]
    wps = 1
    while wps < 8 and slices * wps < 148 * 32:
        wps *= 2
    env.set_kernel_shape(wps, 4)
    pb.apply_bc_at0(env, 0)
    pb.update_acc(env)
    pb.velocity_verlet_step(env, nsteps=w["steps"])
    y2, v2, _, _ = env.get_state()
    assert np.array_equal(y, y2) and np.array_equal(v, v2)
    assert np.array_equal(d, pb.cal_damage(env))
    env.close()


def test_admission_waits_for_footprint():
    big = configs.pmb_cube(dims=(20, 20, 20), steps=3000)
    small = configs.pmb_cube(dims=(8, 8, 8), steps=50)
    # a budget that holds one of them at a time
    with pb.Server(hbm_budget=1) as srv:
        j1 = _submit(srv, big, "fp32c")
        j2 = _submit(srv, small, "fp32c")
        i2 = srv.wait(j2)
        i1 = srv.wait(j1)
        assert i1["state"] == i2["state"] == "done"
        # the second job was only admitted once the first had finished
        assert i2["queue_ms"] > 0.5 * i1["latency_ms"]
        srv.result(j1)
        srv.result(j2)


def test_failed_and_cancelled_jobs():
    w = configs.pmb_cube(dims=(10, 10, 10), steps=50)
    w["materials"][0].general.max_neigh = 20  # families need ~122 members
    long = configs.pmb_cube(dims=(24, 24, 24), steps=200000)
    with pb.Server() as srv:
        jf = _submit(srv, w, "fp32c")
        with pytest.raises(pb.PDError) as e:
            srv.wait(jf)
        assert e.value.status == _abi.PD_ERR_FAMILY_OVERFLOW
        assert srv.poll_state(jf) == "failed"
        jl = _submit(srv, long, "fp32c")
        srv.cancel(jl)
        with pytest.raises(pb.PDError):
            srv.result(jl)
        info = srv.wait(jl)
        assert info["state"] == "cancelled"


def test_serve_stream_reports_latency():
    jobs, arrivals = configs.serving_jobs(8, n_lo=2e3, n_hi=2e4, steps_lo=50, steps_hi=200)
    with pb.Server() as srv:
        recs, summary = pb.serve_stream(srv, jobs, arrivals)
    assert summary["jobs"] == 8 and all(r["state"] == "done" for r in recs)
    assert 0 < summary["latency_ms"]["p50"] <= summary["latency_ms"]["p99"]
    assert summary["bond_updates"] > 0
