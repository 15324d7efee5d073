"""Error behaviour of the C ABI on a GPU: calls made in the wrong state or
with invalid arguments return a status (never abort) and leave a message in
pd_last_error(); a failed call changes nothing, and the environment stays
usable afterwards."""
import ctypes

import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import _abi, configs
from peridyn_b200.environment import GeneralEnvironment

pytestmark = pytest.mark.gpu


def _last_error():
    return _abi.lib().pd_last_error().decode()


def test_create_rejects_bad_device_and_precision():
    L = _abi.lib()
    h = ctypes.c_void_p()
    assert L.pd_env_create(ctypes.byref(h), 4096, 0, 1e-8) == _abi.PD_ERR_ARG
    assert "out of range" in _last_error()
    assert L.pd_env_create(ctypes.byref(h), 0, 7, 1e-8) == _abi.PD_ERR_ARG
    assert "precision" in _last_error()
    assert not h.value


def test_empty_environment_cannot_be_finalized_or_stepped():
    L = _abi.lib()
    h = ctypes.c_void_p()
    assert L.pd_env_create(ctypes.byref(h), 0, 2, 1e-8) == _abi.PD_OK
    try:
        assert L.pd_env_vv_steps(h, 1) == _abi.PD_ERR_STATE
        assert L.pd_env_finalize(h) == _abi.PD_ERR_STATE
        assert "no material blocks" in _last_error()
    finally:
        L.pd_env_destroy(h)


@pytest.mark.parametrize("precision", ["fp64_serial", "fp32c"])
def test_wrong_state_and_bad_arguments_leave_the_environment_usable(precision):
    L = _abi.lib()
    w = configs.pmb_cube(n=6, peak=20.0)
    env = GeneralEnvironment(1, w["materials"], [], [], w["dt"], precision=precision, finalize=False)
    try:
        # stepping before finalize
        assert L.pd_env_vv_steps(env._h, 1) == _abi.PD_ERR_STATE
        assert L.pd_env_finalize(env._h) == _abi.PD_OK
        # a second finalize, a block after finalize
        assert L.pd_env_finalize(env._h) == _abi.PD_ERR_STATE
        assert "already finalized" in _last_error()
        y0, v0, _, _ = env.get_state()
        # negative step count: rejected, nothing moves
        assert L.pd_env_vv_steps(env._h, -1) == _abi.PD_ERR_ARG
        assert L.pd_env_vv_steps(env._h, 0) == _abi.PD_OK
        y1, v1, _, _ = env.get_state()
        assert np.array_equal(y0, y1) and np.array_equal(v0, v1)
        assert env.time_step == 0
        # NULL outputs are skipped, not dereferenced
        assert L.pd_env_get_state(env._h, None, None, None, None) == _abi.PD_OK
        assert L.pd_env_diagnostics(env._h, None) == _abi.PD_ERR_ARG
        # still usable: the same run as a fresh environment's (same kernel
        # shape in the throughput mode)
        ref = pb.Env(1, w["materials"], [], [], w["dt"], precision=precision)
        if precision != "fp64_serial":
            env.set_kernel_shape(1, 4)
            ref.set_kernel_shape(1, 4)
        pb.velocity_verlet_step(env, nsteps=20)
        pb.velocity_verlet_step(ref, nsteps=20)
        for a, b in zip(env.get_state(), ref.get_state()):
            assert np.array_equal(a, b)
        ref.close()
    finally:
        env.close()
