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


def _disk(speed=300.0):
    return configs.disk_impact(radius=3.0e-3, thickness=1.0e-3, spacing=2.5e-4, sphere_radius=1.0e-3, speed=speed)


def _whole_contact(w, precision, nsteps, every):
    env = pb.Env(1, w["materials"], w["contacts"], [], w["dt"], precision=precision)
    env.set_deformed(np.ones(len(w["materials"]), dtype=np.uint8), hold=True)
    pb.update_neighs(env)
    pb.update_acc(env)
    for s in range(nsteps):
        if s and s % every == 0:
            pb.update_neighs(env)
        pb.velocity_verlet_step(env)
    y, v, f, _ = env.get_state()
    broken = sum(int((env._family(b)[0] > 0).sum() - env._family(b)[1].sum()) for b in range(2))
    env.close()
    return y, v, f, broken


def _slabs_contact(w, precision, nsteps, every, nslabs, axis):
    run = SlabRun(w["materials"], [], w["dt"], nslabs, axis=axis, precision=precision, contacts=w["contacts"])
    run.update_neighs()
    run.update_acc()
    for s in range(nsteps):
        if s and s % every == 0:
            run.update_neighs()
        run.step(1)
    y, v, f = run.state()
    run.close()
    return y, v, f


@pytest.mark.parametrize("nslabs,axis", [(2, 0), (3, 1)])
def test_slabs_with_contact_serial_bit_identical(nslabs, axis):
    """Disk struck by a stiff sphere (nonlinear contact), cut into slabs
    across the contact zone: the serial FP64 slabs equal the whole body bit
    for bit, contact neighbour lists rebuilt every 10 steps; by step 100
    ~2,000 bonds under the sphere have broken."""
    w = _disk()
    y0, v0, f0, broken = _whole_contact(w, "fp64_serial", 100, 10)
    assert broken > 0  # the impact breaks bonds under the sphere
    y1, v1, f1 = _slabs_contact(w, "fp64_serial", 100, 10, nslabs, axis)
    assert np.array_equal(y0, y1) and np.array_equal(v0, v1) and np.array_equal(f0, f1)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-4)])
def test_slabs_with_contact_throughput_modes(precision, tol):
    w = _disk()
    x = np.hstack([m.general.x for m in w["materials"]])
    y0, v0, _, _ = _whole_contact(w, precision, 100, 10)
    y1, v1, _ = _slabs_contact(w, precision, 100, 10, 2, 0)
    du = np.linalg.norm((y1 - x) - (y0 - x)) / np.linalg.norm(y0 - x)
    assert du <= tol, du
