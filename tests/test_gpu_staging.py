"""Output staging (pd_env_stage_state / pd_env_stage_read): a snapshot taken
between steps reaches the host unchanged while later steps run, and run!'s
file writes through the staging slots hand the writer the same data as the
synchronous path."""
import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import _abi, configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64_serial", "fp32c"])
def test_staged_snapshot_is_the_state_when_staged(precision):
    w = configs.lps_bar(nx=30, ny=8, nz=8)
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
    pb.apply_bc_at0(env, 0)
    pb.velocity_verlet_step(env, nsteps=20)
    env.stage_state(0)
    y, v, f, _ = env.get_state()
    dmg = pb.cal_damage(env)
    pb.velocity_verlet_step(env, nsteps=30)  # runs while the copy is in flight
    env.stage_state(1)
    s0 = env.read_stage(0)
    assert s0["time_step"] == 20
    assert np.array_equal(s0["position"], y) and np.array_equal(s0["velocity"], v)
    assert np.array_equal(s0["acceleration"], f) and np.array_equal(s0["damage"], dmg)
    s1 = env.read_stage(1)
    assert s1["time_step"] == 50
    assert np.array_equal(s1["position"], env.y)
    with pytest.raises(pb.PDError) as e:
        env.read_stage(0)
    assert e.value.status == _abi.PD_ERR_STATE
    env.close()


def test_run_writes_same_data_staged_and_direct():
    def collect(staged):
        w = configs.lps_bar(nx=24, ny=7, nz=6)
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision="fp32c")
        out = {}
        pb.run(env, 35, pb.DSVelocityVerlet(), filewrite_freq=10, neigh_update_freq=1000,
               writer=lambda name, data: out.__setitem__(name, {k: np.array(v) for k, v in data.items()}),
               staged_io=staged)
        env.close()
        return out

    a, b = collect(False), collect(True)
    assert list(a) == list(b) and len(a) == 7  # start_with, 0, 1, 10, 20, 30, end_with
    for name in a:
        for k in a[name]:
            assert np.array_equal(a[name][k], b[name][k]), (name, k)
