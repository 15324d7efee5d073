"""Slab decomposition on one GPU: the slabs of one body, each its own
environment with two-horizon ghost layers and one halo exchange per step,
against the whole body run as one environment.  Serial FP64 mode:
bit-identical states; throughput modes: within their tolerances
(FP64 1e-10, FP32C 1e-4 relative-L2 of the displacement)."""
import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import _abi, configs
from peridyn_b200.slabs import SlabRun

pytestmark = pytest.mark.gpu


def _whole(w, precision, nsteps):
    env = pb.Env(1, w["materials"], [], w["bcs"], w["dt"], precision=precision)
    env.set_deformed(np.ones(len(w["materials"]), dtype=np.uint8), hold=True)  # as the slabs do
    if w["bcs"]:
        pb.apply_bc_at0(env, 0)
    pb.velocity_verlet_step(env, nsteps=nsteps)
    y, v, f, _ = env.get_state()
    plastic = 0.0
    if w["materials"][0].kind == _abi.PD_MAT_ELASTO_PLASTIC:
        plastic = float(np.abs(env.plastic_strain(0)).max())
    env.close()
    return y, v, f, plastic


def _slabs(w, precision, nsteps, nslabs, axis=0):
    run = SlabRun(w["materials"], w["bcs"], w["dt"], nslabs, axis=axis, precision=precision)
    if w["bcs"]:
        run.apply_bc_at0()
    run.step(nsteps)
    y, v, f = run.state()
    run.close()
    return y, v, f


BUILDERS = {
    "lps_bar": lambda: configs.lps_bar(nx=48, ny=8, nz=8, steps=60),
    "pmb_cube": lambda: configs.pmb_cube(n=14, peak=60.0),
    "ep_bar": lambda: configs.ep_bar(nx=48, ny=8, nz=8, yield_stress=2e5),
}


@pytest.mark.parametrize("name", ["lps_bar", "pmb_cube", "ep_bar"])
@pytest.mark.parametrize("nslabs", [2, 3])
def test_slabs_serial_bit_identical(name, nslabs):
    w = BUILDERS[name]()
    y0, v0, f0, plastic = _whole(w, "fp64_serial", 60)
    if name == "ep_bar":
        assert plastic > 0.0  # bonds yield, so the plastic terms cross the cuts
    y1, v1, f1 = _slabs(w, "fp64_serial", 60, nslabs)
    assert np.array_equal(y0, y1)
    assert np.array_equal(v0, v1)
    assert np.array_equal(f0, f1)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-4)])
@pytest.mark.parametrize("name", ["lps_bar", "pmb_cube"])
def test_slabs_throughput_modes(name, precision, tol):
    w = BUILDERS[name]()
    x = w["materials"][0].general.x
    y0, v0, _, _ = _whole(w, precision, 80)
    y1, v1, _ = _slabs(w, precision, 80, 3)
    du = np.linalg.norm((y1 - x) - (y0 - x)) / np.linalg.norm(y0 - x)
    assert du <= tol, du
