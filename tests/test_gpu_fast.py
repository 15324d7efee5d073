"""Throughput modes (one-pass FP64, FP32-compensated) against the FP64
oracle: relative-L2 error of displacement and velocity after N steps and the
broken-bond mismatch.  Tolerances (stated per test):
  FP64 one-pass: rel-L2 <= 1e-10 (summation order differs from the serial loop)
  FP32C:         rel-L2 <= 1e-4  (the acceptance bound for the FP32 path)
"""
import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import configs, lattice
from tests.cases import bar_with_bcs, ep_cube, random_cloud, self_contact_block

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32c": 1e-4}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _run_pair(oracle, w, precision, nsteps, bc0=True):
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"])
    if bc0:
        ora.apply_bc_at0()
        pb.apply_bc_at0(env, 0)
    for _ in range(nsteps):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=nsteps)
    return env, ora


def _errors(env, ora):
    y, v, f, p = env.get_state()
    x = np.hstack([B.x for B in ora.blocks])
    eu = rel_l2(y - x, ora.y - x)
    ev = rel_l2(v, ora.v)
    mism = 0
    for b, B in enumerate(ora.blocks):
        _, intact = env._family(b)
        mism += int((intact != B.intact.astype(bool)).sum())
    return eu, ev, mism


@pytest.mark.parametrize("layout", ["auto", "explicit"])
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("builder,nsteps", [
    (lambda: configs.pmb_cube(n=12, peak=20.0), 200),
    (lambda: configs.lps_bar(nx=40, ny=10, nz=10), 300),
    (random_cloud, 100),
])
def test_trajectory_error_bound(oracle, precision, builder, nsteps, layout, monkeypatch):
    if layout == "explicit":
        monkeypatch.setenv("PD_FAMILY_LAYOUT", "explicit")
    else:
        monkeypatch.delenv("PD_FAMILY_LAYOUT", raising=False)
    w = builder()
    env, ora = _run_pair(oracle, w, precision, nsteps)
    eu, ev, mism = _errors(env, ora)
    assert eu <= TOL[precision], f"displacement rel-L2 {eu:.3e}"
    assert ev <= TOL[precision], f"velocity rel-L2 {ev:.3e}"
    assert mism == 0
    assert env.time_step == nsteps
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_breaking_mismatch_is_small(oracle, precision):
    w = configs.pmb_cube(n=12, peak=400.0, cs=0.002)
    env, ora = _run_pair(oracle, w, precision, 80, bc0=False)
    eu, ev, mism = _errors(env, ora)
    nbroken = int((ora.blocks[0].family > 0).sum() - ora.blocks[0].intact.sum())
    assert nbroken > 100
    # bonds whose stretch sits within rounding of cs may differ
    assert mism <= max(2, nbroken // 200), f"{mism} of {nbroken} broken bonds differ"
    assert eu <= (1e-8 if precision == "fp64" else 1e-3)
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_lps_breaking_mismatch_is_small(oracle, precision):
    # state-based cube, ~2.8 k of 114 k bonds broken in 80 steps
    w = configs.lps_cube((12, 11, 10), cs=0.002, peak=150.0)
    env, ora = _run_pair(oracle, w, precision, 80, bc0=False)
    eu, ev, mism = _errors(env, ora)
    nbroken = int((ora.blocks[0].family > 0).sum() - ora.blocks[0].intact.sum())
    print(precision, "broken", nbroken, "mismatched", mism, "disp", eu, "vel", ev)
    assert nbroken > 1000
    # measured on B200: no mismatched bond; FP64 1.4e-13 / 5.2e-13, FP32C
    # 1.0e-7 / 3.9e-7 displacement / velocity rel-L2
    assert mism <= max(2, nbroken // 200), f"{mism} of {nbroken} broken bonds differ"
    assert eu <= TOL[precision] and ev <= TOL[precision]
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_multitype_and_tofro(oracle, precision):
    x, vol = lattice.cuboid(14, 6, 6, 1e-3, jitter=1e-5, seed=4)
    t = np.where(x[0] < x[0].mean(), 1, 2).astype(np.int64)
    gen = pb.GeneralMaterial(x.copy(order="F"), np.zeros_like(x, order="F"), x, vol, t, 3.015e-3, max_neigh=200)
    spc = pb.OrdinaryStateBasedSpecific([20e9, 25e9, 30e9], [9e9, 10e9, 12e9], [0.05, 0.05, 0.05], [2000.0, 2500.0])
    mat = pb.PeridynamicsMaterial(gen, spc)
    bcs = [pb.FixBC(x[0] < 2e-3), pb.ToFroBC(x[0] > 12e-3, [2.0, 0.3, 0.0], 40, applyafter=10)]
    w = {"materials": [mat], "contacts": [], "bcs": bcs, "dt": 2e-8}
    env, ora = _run_pair(oracle, w, precision, 150)
    eu, ev, mism = _errors(env, ora)
    assert eu <= TOL[precision] and ev <= TOL[precision] and mism == 0
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_chunked_equals_single_run(precision):
    w = configs.lps_bar(nx=30, ny=8, nz=8)
    e1 = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
    e2 = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
    for e in (e1, e2):
        pb.apply_bc_at0(e, 0)
    pb.velocity_verlet_step(e1, nsteps=60)
    for _ in range(6):
        pb.velocity_verlet_step(e2, nsteps=10)
        e2.get_state()  # reads do not perturb the device state
    s1, s2 = e1.get_state(), e2.get_state()
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    e1.close()
    e2.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_contact_impact_fast(oracle, precision):
    w = configs.disk_impact(radius=2.0e-3, thickness=1.0e-3, spacing=2.5e-4, sphere_radius=0.75e-3, speed=150.0,
                            cs=0.003)
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"])
    ora.update_acc()
    pb.update_acc(env)
    for _ in range(60):
        ora.update_neighs()
        pb.update_neighs(env)
        ora.vv_step()
        pb.velocity_verlet_step(env)
    eu, ev, mism = _errors(env, ora)
    print(f"\ncontact impact {precision}: displacement {eu:.3e}, velocity {ev:.3e}, mismatched {mism}")
    assert eu <= (1e-9 if precision == "fp64" else TOL["fp32c"]), eu
    assert mism == 0
    env.close()


@pytest.mark.parametrize("ordered", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_self_contact_fast(oracle, precision, ordered):
    w, families = self_contact_block(oracle, ordered=ordered)
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision, families=families)
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"], families=families)
    for _ in range(8):
        ora.update_neighs()
        pb.update_neighs(env)
        assert np.array_equal(env.contact_neighs(0), ora.contacts[0].neighs)
        ora.vv_step()
        pb.velocity_verlet_step(env)
    eu, ev, mism = _errors(env, ora)
    assert eu <= TOL[precision], eu
    assert ev <= (1e-9 if precision == "fp64" else 1e-3), ev
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_rigid_gate_fast(precision):
    w = configs.pmb_cube(n=8, peak=0.0)
    w["materials"][0].general.velocity[0] = 3.0
    env = pb.Env(1, w["materials"], [], [], w["dt"], precision=precision)
    pb.velocity_verlet_step(env, nsteps=10)
    assert not env.deformed()[0]
    assert np.all(env.f == 0.0)
    env.close()


def test_update_acc_fast_matches_oracle(oracle):
    # One force evaluation of an LPS bar under a random 1e-6 m displacement
    # field (no smooth deformation): the dilatation and the bond terms of
    # each particle are sums of terms of both signs that cancel to a small
    # remainder, so the relative error of f and theta in FP32 is larger than
    # on a trajectory, where the 1e-4 bound holds.  FP32C is held to 2e-4
    # here, the one-pass FP64 path to 1e-12.
    w = configs.lps_bar(nx=24, ny=7, nz=6)
    for precision, tol in (("fp64", 1e-12), ("fp32c", 2e-4)):
        env = pb.Env(1, w["materials"], [], [], w["dt"], precision=precision)
        ora = oracle.OracleEnv(w["materials"], [], [], w["dt"])
        rng = np.random.default_rng(2)
        y = ora.y + rng.normal(0.0, 1e-6, size=ora.y.shape)
        ora.y[:] = y
        env.set_state(y=y)
        ora.update_acc()
        pb.update_acc(env)
        assert rel_l2(env.f, ora.f) <= tol
        assert np.allclose(env.theta(0), ora.blocks[0].theta, rtol=tol, atol=tol * np.abs(ora.blocks[0].theta).max())
        env.close()


def _tofro_bar():
    x, vol = lattice.cuboid(14, 6, 6, 1e-3, jitter=1e-5, seed=4)
    gen = pb.GeneralMaterial(x.copy(order="F"), np.zeros_like(x, order="F"), x, vol, np.ones(x.shape[1], np.int64),
                             3.015e-3, max_neigh=200)
    mat = pb.PeridynamicsMaterial(gen, pb.OrdinaryStateBasedSpecific([20e9], [9e9], [0.05], [2000.0]))
    bcs = [pb.FixBC(x[0] < 2e-3), pb.ToFroBC(x[0] > 12e-3, [2.0, 0.3, 0.0], 40, applyafter=10)]
    return {"materials": [mat], "contacts": [], "bcs": bcs, "dt": 2e-8}


def _small_impact():
    return configs.disk_impact(radius=3.0e-3, thickness=1.0e-3, spacing=2.5e-4, sphere_radius=1.0e-3, speed=300.0)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("builder", [_tofro_bar, lambda: configs.batched_cubes(nspec=6, edge_lo=5, edge_hi=9),
                                     _small_impact])
def test_graph_replay_matches_direct_launches(precision, builder, monkeypatch):
    # graph replays of 32 steps (between BC direction flips, gate kernels
    # included while a block is undeformed; with contact, between neighbour
    # updates, the contact kernels captured with the step) against one
    # launch per kernel
    w = builder()

    def run():
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
        if w["bcs"]:
            pb.apply_bc_at0(env, 0)
        if w["contacts"]:
            pb.update_neighs(env)
            pb.update_acc(env)
        pb.velocity_verlet_step(env, nsteps=150)
        if w["contacts"]:
            pb.update_neighs(env)  # new lists: the captured contact steps are re-captured
        pb.velocity_verlet_step(env, nsteps=75)
        out = env.get_state(), [env._family(b)[1] for b in range(len(w["materials"]))], env.deformed()
        env.close()
        return out

    monkeypatch.setenv("PD_NO_GRAPHS", "1")
    (s1, i1, d1) = run()
    monkeypatch.delenv("PD_NO_GRAPHS")
    (s2, i2, d2) = run()
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    for a, b in zip(i1, i2):
        assert np.array_equal(a, b)
    assert np.array_equal(d1, d2)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_rigid_gate_fast_long_run(precision):
    # long enough for graph replays: the gate stays in every replayed step
    w = configs.pmb_cube(n=8, peak=0.0)
    w["materials"][0].general.velocity[0] = 3.0
    env = pb.Env(1, w["materials"], [], [], w["dt"], precision=precision)
    pb.velocity_verlet_step(env, nsteps=100)
    assert not env.deformed()[0]
    assert np.all(env.f == 0.0)
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("kind", ["delta", "scalefixwait", "container"])
def test_scaling_and_container_bcs_fast(oracle, precision, kind):
    w = bar_with_bcs(kind)
    env, ora = _run_pair(oracle, w, precision, 95)
    eu, ev, mism = _errors(env, ora)
    assert eu <= TOL[precision], f"displacement rel-L2 {eu:.3e}"
    assert ev <= TOL[precision], f"velocity rel-L2 {ev:.3e}"
    assert mism == 0
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("case", ["bar_2warps", "batch16_1warp", "batch16_2warps"])
def test_persistent_chunks_match_graph_replays(precision, case, monkeypatch):
    # PD_PERSIST=1: flip-free runs of a deformed problem in one cooperative
    # launch with grid barriers; same shape, so the same numbers.  The
    # 16-specimen batch has more slice groups than the device holds blocks
    # at once, so each block walks several groups per phase.
    from peridyn_b200 import _abi

    if case == "bar_2warps":
        w, wps = configs.lps_bar(nx=30, ny=8, nz=8), 2
    else:
        w, wps = configs.batched_cubes(nspec=16), 1 if case == "batch16_1warp" else 2

    def run(persist):
        if persist:
            monkeypatch.setenv("PD_PERSIST", "1")
        else:
            monkeypatch.delenv("PD_PERSIST", raising=False)
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
        env.set_kernel_shape(wps, (4 if wps == 1 else 2) if precision == "fp32c" else 1)
        if w["bcs"]:
            pb.apply_bc_at0(env, 0)
        pb.velocity_verlet_step(env, nsteps=40)   # deforms: the gate drops out
        n0 = _abi.kernel_launches()
        pb.velocity_verlet_step(env, nsteps=120)  # persistent when enabled
        launches = _abi.kernel_launches() - n0
        out = env.get_state()
        env.close()
        return out, launches

    (s0, l0), (s1, l1) = run(False), run(True)
    assert l1 < l0 // 4  # one cooperative launch instead of graph replays of 120 steps
    for a, b in zip(s0, s1):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
@pytest.mark.parametrize("builder", [
    lambda: configs.lps_bar(nx=30, ny=8, nz=8),
    lambda: configs.ep_bar(nx=30, ny=8, nz=8, yield_stress=2e5),
])
def test_dependent_launch_is_bit_identical(builder, precision, monkeypatch):
    # the bond kernels launched with programmatic stream serialization
    # (default) and as ordinary launches (PD_NO_PDL=1): same numbers, in
    # graph replays and direct launches alike
    w = builder()

    def run(pdl):
        if pdl:
            monkeypatch.delenv("PD_NO_PDL", raising=False)
        else:
            monkeypatch.setenv("PD_NO_PDL", "1")
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
        pb.apply_bc_at0(env, 0)
        pb.velocity_verlet_step(env, nsteps=5)    # direct launches
        pb.velocity_verlet_step(env, nsteps=100)  # graph replays
        out = env.get_state() + (env.num_bonds(),)
        env.close()
        return out

    for a, b in zip(run(True), run(False)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64_serial", "fp64", "fp32c"])
def test_held_undeformed_block_gets_no_forces(precision):
    # pd_env_set_deformed(..., hold): a block held undeformed is skipped by
    # the force kernels (its gate flag is read, since not every block has
    # deformed), the other block is not: with no force the held block's
    # velocities stay exactly as they started, in direct launches and in
    # graph replays alike
    w = configs.batched_cubes(nspec=2, edge_lo=6, edge_hi=9)
    n0 = w["materials"][0].general.n
    env = pb.Env(1, w["materials"], [], [], w["dt"], precision=precision)
    env.set_deformed(np.array([1, 0], dtype=np.uint8), hold=True)
    pb.velocity_verlet_step(env, nsteps=5)  # (FP32C keeps v in FP32: compare from here)
    _, v0, _, _ = env.get_state()
    pb.velocity_verlet_step(env, nsteps=70)
    _, v1, _, _ = env.get_state()
    env.close()
    assert np.array_equal(v1[:, n0:], v0[:, n0:])
    assert not np.array_equal(v1[:, :n0], v0[:, :n0])


def _two_type_block():
    x, vol = lattice.cuboid(16, 9, 8, 1.0e-3, jitter=2e-5, seed=9)
    t = np.where(x[0] < x[0].mean(), 1, 2).astype(np.int64)
    gen = pb.GeneralMaterial(x.copy(order="F"), lattice.gaussian_pulse(x, 40.0, 2e-3), x, vol, t, 3.015e-3,
                             max_neigh=200)
    spc = pb.OrdinaryStateBasedSpecific([20e9, 25e9, 30e9], [9e9, 10e9, 12e9], [0.004, 0.003, 0.005],
                                        [2000.0, 2500.0])
    return {"materials": [pb.PeridynamicsMaterial(gen, spc)], "contacts": [], "bcs": [], "dt": 2e-8}


@pytest.mark.parametrize("shape", [(4, 2), (4, 4), (8, 2), (8, 4)])
@pytest.mark.parametrize("builder", [
    lambda: configs.lps_bar(nx=30, ny=8, nz=8),
    lambda: configs.pmb_cube(n=14, peak=60.0),
    _two_type_block,
    lambda: configs.batched_cubes(nspec=5, edge_lo=6, edge_hi=11),
])
def test_record_staging_is_bit_identical(builder, shape):
    """The staged kernels (neighbour records copied to shared memory by bulk
    asynchronous copies) do the same arithmetic in the same order as the
    global-load kernels: identical states and broken-bond sets."""
    w = builder()

    def run(staging):
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision="fp32c")
        env.set_kernel_shape(*shape)
        env.set_record_staging(staging)
        if w["bcs"]:
            pb.apply_bc_at0(env, 0)
        pb.velocity_verlet_step(env, nsteps=120)
        st = env.record_staging()
        out = env.get_state(), [env._family(b)[1] for b in range(len(w["materials"]))]
        env.close()
        return out, st

    (s1, i1), st1 = run(0)
    (s2, i2), st2 = run(1)
    assert not st1["staged"]
    assert st2["staged"] and st2["slices"] > 0 and 0 < st2["max_records"] <= 2048
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    for a, b in zip(i1, i2):
        assert np.array_equal(a, b)
    assert sum(int((~i).sum()) for i in i1) >= 0


def test_record_staging_autotuned_bar_matches_oracle(oracle):
    w = configs.lps_bar(nx=40, ny=10, nz=10)
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision="fp32c")
    env.set_record_staging(2)
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"])
    ora.apply_bc_at0()
    pb.apply_bc_at0(env, 0)
    for _ in range(200):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=200)
    eu, ev, mism = _errors(env, ora)
    assert eu <= TOL["fp32c"], eu
    assert env.record_staging()["slices"] > 0
    env.close()


@pytest.mark.parametrize("shape", [(4, 2), (8, 4)])
def test_slice_swizzle_is_bit_identical(shape, monkeypatch):
    # one-slice-per-block kernels walk slices in SM-grouped order by
    # default; the order of blocks changes no arithmetic
    w = configs.lps_bar(nx=60, ny=10, nz=10)

    def run():
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision="fp32c")
        env.set_kernel_shape(*shape)
        pb.apply_bc_at0(env, 0)
        pb.velocity_verlet_step(env, nsteps=100)
        out = env.get_state(), env._family(0)[1]
        env.close()
        return out

    monkeypatch.setenv("PD_SWIZZLE", "0")
    s1, i1 = run()
    monkeypatch.delenv("PD_SWIZZLE")
    s2, i2 = run()
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    assert np.array_equal(i1, i2)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("builder", [lambda: ep_cube(5e6), lambda: ep_cube(2e6, ntypes=2),
                                     lambda: ep_cube(5e6, peak=300.0, cs=0.003), lambda: configs.ep_bar(nx=40)])
def test_elasto_plastic_fast(oracle, precision, builder):
    """Throughput-mode elasto-plastic solid (td_norm2 pass with bond
    breaking, both visits' terms per bond, per-slot plastic strain) against
    the serial oracle: displacement, velocity, plastic strain and bonds."""
    w = builder()
    bc0 = bool(w["bcs"])
    nsteps = 40
    env, ora = _run_pair(oracle, w, precision, nsteps, bc0=bc0)
    eu, ev, mism = _errors(env, ora)
    tol = TOL[precision]
    assert eu <= tol, eu
    assert ev <= (1e-9 if precision == "fp64" else 1e-3), ev
    B = ora.blocks[0]
    edp = env.plastic_strain(0)
    fam = B.family > 0
    assert np.abs(B.edp[fam]).max() > 0.0
    assert rel_l2(edp[fam], B.edp[fam]) <= (1e-8 if precision == "fp64" else 2e-3)
    if precision == "fp64":
        assert mism == 0
    env.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_elasto_plastic_fast_graphs_match_direct(precision, monkeypatch):
    # graph replays alternate the plastic strain buffers like direct launches
    w = configs.ep_bar(nx=30)

    def run():
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
        pb.apply_bc_at0(env, 0)
        pb.velocity_verlet_step(env, nsteps=101)
        out = env.get_state(), env._family(0)[1], env.plastic_strain(0)
        env.close()
        return out

    monkeypatch.setenv("PD_NO_GRAPHS", "1")
    s1, i1, e1 = run()
    monkeypatch.delenv("PD_NO_GRAPHS")
    s2, i2, e2 = run()
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    assert np.array_equal(i1, i2)
    assert np.array_equal(e1, e2)


def test_pipe_peaks_are_physical():
    """pd_pipe_peaks (the compute-side roofline denominators): every rate
    positive and below what the SMs could do at 2.2 GHz (128 FP32 lanes, 16
    MUFU lanes and 4 issuing sub-partitions per SM)."""
    import torch

    from peridyn_b200 import _abi

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    r = _abi.pipe_peaks(0)
    print(r)
    clk = 2.2e9
    assert 0 < r["ffma_lane_ops_per_s"] <= sms * 128 * clk
    assert 0 < r["ffma2_lane_fmas_per_s"] <= 2 * sms * 128 * clk
    for k in ("sqrt_approx_lane_ops_per_s", "rcp_approx_lane_ops_per_s"):
        assert 0 < r[k] <= sms * 32 * clk
    assert 0 < r["ffma_lop3_warp_instr_per_s"] <= sms * 4 * clk
    # a full grid of independent chains keeps the FMA pipe busy
    assert r["ffma_lane_ops_per_s"] >= 0.5 * sms * 128 * 1.0e9


@pytest.mark.parametrize("shape", [(4, 2), (4, 4), (8, 4)])
def test_shattered_cube_walks_agree(shape):
    """A cube shattered by a 3000 m/s pulse (over 30 % of its bonds broken in
    200 steps): the global-load stencil walk (offsets read one group ahead)
    and the staged walk give the same states and broken-bond sets, bit for
    bit, with most of the bond bits cleared while the walks run."""
    w = configs.pmb_cube(n=14, peak=3000.0)

    def run(staging):
        env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision="fp32c")
        env.set_kernel_shape(*shape)
        env.set_record_staging(staging)
        b0 = env.num_bonds()
        pb.velocity_verlet_step(env, nsteps=200)
        out = env.get_state(), env._family(0)[1], 1.0 - env.num_bonds() / b0
        env.close()
        return out

    s1, i1, broken = run(0)
    s2, i2, _ = run(1)
    print("broken fraction", broken)
    assert broken > 0.3
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    assert np.array_equal(i1, i2)
