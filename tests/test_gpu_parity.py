"""Parity of the CUDA serial-order FP64 path with the CPU oracle: bit-exact
families, weighted volumes, forces, broken-bond sets, trajectories,
boundary conditions, contacts, QSDrag and damage."""
import ctypes

import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import _abi, configs, lattice
from tests.cases import bar_with_bcs, ep_cube, random_cloud, self_contact_block

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["auto", "explicit"])
def layout(request, monkeypatch):
    """Bond storage form chosen at finalize: per-slice stencil where the
    offsets allow it ("auto") or explicit indices everywhere."""
    if request.param == "explicit":
        monkeypatch.setenv("PD_FAMILY_LAYOUT", "explicit")
    else:
        monkeypatch.delenv("PD_FAMILY_LAYOUT", raising=False)
    return request.param


def _check_layout(env, layout):
    st = env.layout()
    if layout == "explicit":
        assert st["stencil_slices"] == 0
    else:
        assert st["stencil_slices"] > 0


def _pair(oracle, w, precision="fp64_serial", families=None):
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision, families=families)
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"], families=families)
    return env, ora


def _assert_state_equal(env, ora, what=""):
    y, v, f, p = env.get_state()
    assert np.array_equal(y, ora.y), f"y differs {what}"
    assert np.array_equal(v, ora.v), f"v differs {what}"
    assert np.array_equal(f, ora.f), f"f differs {what}"
    assert np.array_equal(p, ora.p), f"p differs {what}"


def _assert_bonds_equal(env, ora):
    for b, B in enumerate(ora.blocks):
        fam, intact = env._family(b)
        assert np.array_equal(fam, B.family)
        assert np.array_equal(intact, B.intact.astype(bool))


def small_bar():
    return configs.lps_bar(nx=24, ny=7, nz=6, steps=40)


def multitype_block():
    x, vol = lattice.cuboid(9, 8, 7, 1.0e-3, jitter=2e-5, seed=9)
    t = np.where(x[0] < x[0].mean(), 1, 2).astype(np.int64)
    gen = pb.GeneralMaterial(x.copy(order="F"), lattice.gaussian_pulse(x, 5.0, 2e-3), x, vol, t, 3.015e-3,
                             max_neigh=200)
    spc = pb.OrdinaryStateBasedSpecific([20e9, 25e9, 30e9], [9e9, 10e9, 12e9], [0.004, 0.003, 0.005],
                                        [2000.0, 2500.0])
    mat = pb.PeridynamicsMaterial(gen, spc, name="two-type")
    return {"materials": [mat], "contacts": [], "bcs": [], "dt": 2e-8, "steps": 20}


@pytest.mark.parametrize("builder", [lambda: configs.pmb_cube(n=11), small_bar, multitype_block,
                                     lambda: configs.batched_cubes(nspec=5, edge_lo=5, edge_hi=9)])
def test_family_weighted_volume_bit_exact(oracle, builder, layout):
    w = builder()
    env, ora = _pair(oracle, w)
    _check_layout(env, layout)
    _assert_bonds_equal(env, ora)
    for b, B in enumerate(ora.blocks):
        assert np.array_equal(w["materials"][b].general.weighted_volume, B.m)
    assert np.array_equal(env.intact0, ora.intact0)
    assert np.array_equal(env.mass, ora.mass) and np.array_equal(env.density, ora.density)
    env.close()


def test_knife_edge_exact_lattice_counts(oracle):
    # horizon = 3 * spacing on x = i * spacing: the |v|^2 = 9 bonds sit on
    # the d^2 < h^2 edge; only identical FP64 arithmetic agrees on them
    w = configs.lps_bar(nx=40, ny=9, nz=9)
    env, ora = _pair(oracle, w)
    _assert_bonds_equal(env, ora)
    env.close()


@pytest.mark.parametrize("builder", [lambda: configs.pmb_cube(n=10), small_bar, multitype_block])
def test_update_acc_bit_exact_with_breaking(oracle, builder, layout):
    w = builder()
    env, ora = _pair(oracle, w)
    _check_layout(env, layout)
    _update_acc_with_breaking(env, ora)
    env.close()


def test_update_acc_disordered_cloud(oracle):
    w = random_cloud()
    env, ora = _pair(oracle, w)
    st = env.layout()
    assert st["stencil_slices"] < st["slices"] // 4
    _update_acc_with_breaking(env, ora)
    for _ in range(10):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=10)
    _assert_state_equal(env, ora)
    _assert_bonds_equal(env, ora)
    env.close()


def _update_acc_with_breaking(env, ora):
    rng = np.random.default_rng(1)
    y = ora.y + rng.normal(0.0, 4e-6, size=ora.y.shape)
    ora.y[:] = y
    env.set_state(y=y)
    before = sum(int(B.intact.sum()) for B in ora.blocks)
    ora.update_acc()
    pb.update_acc(env)
    after = sum(int(B.intact.sum()) for B in ora.blocks)
    assert after < before  # the perturbation breaks bonds
    _assert_state_equal(env, ora)
    _assert_bonds_equal(env, ora)
    for b, B in enumerate(ora.blocks):
        if B.kind == 1:
            assert np.array_equal(env.theta(b), B.theta)
    assert np.array_equal(pb.cal_damage(env), ora.damage())


@pytest.mark.parametrize("builder,nsteps", [(lambda: configs.pmb_cube(n=10, peak=60.0), 60), (small_bar, 60),
                                            (multitype_block, 30)])
def test_velocity_verlet_trajectory_bit_exact(oracle, builder, nsteps, layout):
    w = builder()
    env, ora = _pair(oracle, w)
    _check_layout(env, layout)
    ora.update_acc()
    pb.update_acc(env)
    ora.apply_bc_at0()
    pb.apply_bc_at0(env, 0)
    for k in range(nsteps):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=nsteps)
    assert env.time_step == ora.time_step == nsteps
    _assert_state_equal(env, ora, f"after {nsteps} steps")
    _assert_bonds_equal(env, ora)
    assert np.array_equal(pb.cal_damage(env), ora.damage())
    env.close()


def test_bond_breaking_trajectory_bit_exact(oracle):
    # strong pulse and low critical stretch: bonds break during the run
    w = configs.pmb_cube(n=12, peak=400.0, cs=0.002)
    env, ora = _pair(oracle, w)
    for _ in range(80):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=80)
    assert ora.damage().max() > 0
    _assert_state_equal(env, ora)
    _assert_bonds_equal(env, ora)
    env.close()


def test_lps_bond_breaking_trajectory_bit_exact(oracle):
    # state-based cube, low critical stretch, 150 m/s pulse: ~2.8 k of 114 k
    # bonds break in 80 steps; the dilatation of each step uses the previous
    # step's intact bonds (peri.jl:155-172), the force pass breaks
    w = configs.lps_cube((12, 11, 10), cs=0.002, peak=150.0)
    env, ora = _pair(oracle, w)
    for _ in range(80):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=80)
    assert int((ora.blocks[0].family > 0).sum() - ora.blocks[0].intact.sum()) > 1000
    _assert_state_equal(env, ora)
    _assert_bonds_equal(env, ora)
    assert np.array_equal(pb.cal_damage(env), ora.damage())
    env.close()


def test_rigid_translation_gate(oracle):
    w = configs.pmb_cube(n=8, peak=0.0)
    mat = w["materials"][0]
    mat.general.velocity[0] = 3.0  # uniform velocity: rigid motion
    env, ora = _pair(oracle, w)
    for _ in range(10):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=10)
    assert not env.deformed()[0] and not ora.blocks[0].deformed
    assert np.all(env.f == 0.0)
    _assert_state_equal(env, ora)
    env.close()


def test_tofro_bc_direction_flips(oracle):
    x, vol = lattice.cuboid(12, 5, 5, 1e-3)
    gen = pb.GeneralMaterial(x.copy(order="F"), np.zeros_like(x, order="F"), x, vol,
                             np.ones(x.shape[1], dtype=np.int64), 3.015e-3, max_neigh=200)
    mat = pb.PeridynamicsMaterial(gen, pb.BondBasedSpecific([10e9], [0.05], [2000.0]))
    bcs = [pb.FixBC(x[0] < 2e-3), pb.ToFroBC(x[0] > 10e-3, [3.0, 0.5, 0.0], 7, applyafter=3)]
    w = {"materials": [mat], "contacts": [], "bcs": bcs, "dt": 1e-8}
    env, ora = _pair(oracle, w)
    ora.apply_bc_at0()
    pb.apply_bc_at0(env, 0)
    for _ in range(30):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=30)
    _assert_state_equal(env, ora)
    env.close()


def test_qsdrag_bit_exact(oracle):
    w = small_bar()
    env, ora = _pair(oracle, w)
    ora.apply_bc_at0()
    pb.apply_bc_at0(env, 0)
    for _ in range(5):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=5)
    solver = pb.QSDrag(1e-8, 1e5, max_iter=15, x_tol=1e-12, f_tol=1e-3)
    it_o = ora.minimize(solver.step_size, solver.drag, solver.max_iter, solver.x_tol, solver.f_tol)
    it_g = pb.minimize(env, solver)
    assert it_o == it_g
    _assert_state_equal(env, ora)
    env.close()


def test_device_pointer_entry_point(oracle):
    torch = pytest.importorskip("torch")
    w = small_bar()
    env, ora = _pair(oracle, w)
    rng = np.random.default_rng(5)
    y = np.asfortranarray(ora.y + rng.normal(0.0, 2e-6, size=ora.y.shape))
    f0 = np.asfortranarray(rng.normal(0.0, 1.0, size=ora.y.shape))
    # reference: f_ .+= contributions (force_density_T! accumulates into f)
    ora.y[:] = y
    ora.f[:] = f0
    ora.force_density_T(ora.blocks[0])
    yd = torch.from_numpy(np.ascontiguousarray(y.T)).cuda()  # (N,3) row-major == 3xN column-major
    fd = torch.from_numpy(np.ascontiguousarray(f0.T)).cuda()
    st = _abi.lib().pd_force_density_device(env._h, 0, ctypes.c_void_p(fd.data_ptr()),
                                            ctypes.c_void_p(yd.data_ptr()), None)
    _abi.check(st)
    f = fd.cpu().numpy().T
    assert np.array_equal(f, ora.f)
    _assert_bonds_equal(env, ora)
    env.close()


def _impact(n_scale=1.0):
    return configs.disk_impact(radius=2.0e-3 * n_scale, thickness=1.0e-3, spacing=2.5e-4, sphere_radius=0.75e-3,
                               speed=150.0, cs=0.003, steps=60)


def test_contact12_neighbours_and_forces_bit_exact(oracle):
    w = _impact()
    env, ora = _pair(oracle, w)
    ora.update_acc()
    pb.update_acc(env)
    touched = 0
    for step in range(60):
        ora.update_neighs()
        pb.update_neighs(env)
        assert np.array_equal(env.contact_neighs(0), ora.contacts[0].neighs), f"neighs at step {step}"
        touched += int((ora.contacts[0].neighs > 0).sum())
        ora.vv_step()
        pb.velocity_verlet_step(env)
    assert touched > 0
    _assert_state_equal(env, ora)
    _assert_bonds_equal(env, ora)
    env.close()


@pytest.mark.parametrize("ordered", [False, True])
def test_contact11_self_contact_bit_exact(oracle, layout, ordered):
    """Both self-contact searches: the reference's merge walk (at most the
    first family member) and the ordered search (every qualifying member,
    so several rows per particle and reverse lists with several sources)."""
    w, families = self_contact_block(oracle, ordered=ordered)
    env, ora = _pair(oracle, w, families=families)
    _check_layout(env, layout)
    hits = multi = 0
    for _ in range(8):
        ora.update_neighs()
        pb.update_neighs(env)
        assert np.array_equal(env.contact_neighs(0), ora.contacts[0].neighs)
        hits += int((ora.contacts[0].neighs > 0).sum())
        multi += int((ora.contacts[0].neighs[1] > 0).sum())
        ora.vv_step()
        pb.velocity_verlet_step(env)
    assert hits > 0
    assert (multi > 0) == ordered
    _assert_state_equal(env, ora)
    env.close()


def test_run_cadence_matches(oracle):
    w = small_bar()
    env, ora = _pair(oracle, w)
    pb.run(env, 23, pb.DSVelocityVerlet(), filewrite_freq=4, neigh_update_freq=1000)
    ora.run(23, filewrite_freq=4, neigh_update_freq=1000)
    _assert_state_equal(env, ora)
    env.close()


def test_full_size_lps_bar_bit_exact(oracle):
    # the 100x20x20 tensile bar at full size, 12 steps
    w = configs.lps_bar()
    env, ora = _pair(oracle, w)
    ora.apply_bc_at0()
    pb.apply_bc_at0(env, 0)
    for _ in range(12):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=12)
    _assert_state_equal(env, ora)
    _assert_bonds_equal(env, ora)
    env.close()


def test_family_overflow_is_reported():
    x, vol = lattice.cuboid(7, 7, 7, 1.0)
    gen = pb.GeneralMaterial(x.copy(order="F"), np.zeros_like(x, order="F"), x, vol, np.ones(x.shape[1], np.int64),
                             3.015, max_neigh=122)
    mat = pb.PeridynamicsMaterial(gen, pb.BondBasedSpecific([1.0], [0.1], [1.0]))
    with pytest.raises(pb.PDError) as e:
        pb.Env(1, [mat], [], [], 1e-3)
    assert e.value.status == _abi.PD_ERR_FAMILY_OVERFLOW


def test_family_at_the_max_neigh_boundary(oracle):
    # 122 neighbours in the exact lattice's interior: max_neigh = 122 is one
    # short (the overflow above, and the oracle's BoundsError), 123 builds
    # the same family as the oracle
    x, vol = lattice.cuboid(7, 7, 7, 1.0)
    with pytest.raises(IndexError):
        oracle.cal_family(x, 3.015, 122)
    fam_ref, _ = oracle.cal_family(x, 3.015, 123)
    gen = pb.GeneralMaterial(x.copy(order="F"), np.zeros_like(x, order="F"), x, vol, np.ones(x.shape[1], np.int64),
                             3.015, max_neigh=123)
    mat = pb.PeridynamicsMaterial(gen, pb.BondBasedSpecific([1.0], [0.1], [1.0]))
    env = pb.Env(1, [mat], [], [], 1e-3)
    fam, intact = env._family(0)
    assert int((fam > 0).sum(axis=0).max()) == 122
    assert np.array_equal(fam, fam_ref) and np.array_equal(intact, fam > 0)
    env.close()


@pytest.mark.parametrize("kind", ["delta", "scalefixwait", "container"])
def test_scaling_and_container_bcs_bit_exact(oracle, kind):
    # DeltaScaleBC.jl, ScaleFixWaitBC.jl (check! every 10 steps), ContainerBC.jl
    w = bar_with_bcs(kind)
    env, ora = _pair(oracle, w)
    ora.apply_bc_at0()
    pb.apply_bc_at0(env, 0)
    ora.update_acc()
    pb.update_acc(env)
    for _ in range(45):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=25)
    pb.velocity_verlet_step(env, nsteps=20)
    _assert_state_equal(env, ora, kind)
    _assert_bonds_equal(env, ora)
    it_o = ora.minimize(1e-7, 10.0, max_iter=5)
    it_g = pb.minimize(env, pb.QSDrag(1e-7, 10.0, max_iter=5))
    assert it_o == it_g
    _assert_state_equal(env, ora, kind + " after QSDrag")
    env.close()


@pytest.mark.parametrize("builder", [lambda: ep_cube(5e6), lambda: ep_cube(2e6, ntypes=2),
                                     lambda: ep_cube(5e6, peak=300.0, cs=0.003)])
def test_elasto_plastic_bit_exact(oracle, builder, layout):
    # td_norm2 pass, asymmetric bond terms (each end's own edp and td_norm2)
    w = builder()
    env, ora = _pair(oracle, w)
    _check_layout(env, layout)
    for _ in range(40):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=40)
    _assert_state_equal(env, ora)
    _assert_bonds_equal(env, ora)
    B = ora.blocks[0]
    assert np.abs(B.edp).max() > 0.0
    assert np.array_equal(env.plastic_strain(0), B.edp)
    assert np.array_equal(env.theta(0), B.theta)
    env.close()


def test_elasto_plastic_serial_plastic_strain_export(oracle):
    w = ep_cube(5e6, n=6)
    env, ora = _pair(oracle, w)
    for _ in range(10):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=10)
    assert np.array_equal(env.plastic_strain(0), ora.blocks[0].edp)
    env.close()
