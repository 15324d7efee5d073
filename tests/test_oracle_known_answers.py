"""Pins the CPU oracle (oracle/) with analytical known answers derived from
the reference's formulas, and checks the GPU algorithm's summation order
on the CPU.  The reference ships no tests or fixtures of its own."""
import math

import numpy as np
import pytest

from peridyn_b200 import (BondBasedSpecific, GeneralMaterial, NonLinearSpringContactModel, OrdinaryStateBasedSpecific,
                          PeridynamicsMaterial, configs, julia_pow_int, lattice, make_matrix)
from tests import gather_order


def lattice_block(n, spacing, horizon_factor, kind="pmb", stretch=1.0, jitter=0.0, cs=0.5, centered=True, seed=1,
                  K=1.0e9, G=0.6e9, rho=1000.0):
    x, vol = lattice.cuboid(n, n, n, spacing, jitter=jitter, seed=seed, centered=centered)
    y = np.asfortranarray(stretch * x)
    v = np.zeros_like(x, order="F")
    gen = GeneralMaterial(y, v, x, vol, np.ones(x.shape[1], dtype=np.int64), horizon_factor * spacing,
                          max_neigh=200)
    spc = BondBasedSpecific([K], [cs], [rho]) if kind == "pmb" else OrdinaryStateBasedSpecific([K], [G], [cs], [rho])
    return PeridynamicsMaterial(gen, spc)


def integer_vectors_below(r2):
    r = int(math.ceil(math.sqrt(r2)))
    cnt = 0
    for i in range(-r, r + 1):
        for j in range(-r, r + 1):
            for k in range(-r, r + 1):
                if 0 < i * i + j * j + k * k < r2:
                    cnt += 1
    return cnt


def test_fld_matches_julia_semantics(oracle):
    L = oracle.lib()
    # Julia: fld(1.0, 0.1) == 9.0 (exact remainder semantics), fld(7.0, 2.0) == 3.0
    assert L.or_fld(1.0, 0.1) == 9.0
    assert L.or_fld(7.0, 2.0) == 3.0
    assert L.or_fld(-1.0, 3.0) == -1.0
    assert L.or_fld(6.0, 3.0) == 2.0
    assert L.or_fld(0.0, 3.0) == 0.0


def test_pow_restatements_agree(oracle):
    rng = np.random.default_rng(0)
    L = oracle.lib()
    for x in rng.uniform(0.0, 3.0, 200):
        for n in (1, 2, 3, 4, 5, 7):
            assert julia_pow_int(float(x), n) == L.or_pow(float(x), float(n))
    assert julia_pow_int(0.3, 2) == 0.3 * 0.3


def test_make_matrix():
    m = make_matrix([1.0, 2.0, 3.0])
    assert m.shape == (2, 2) and m[0, 0] == 1 and m[0, 1] == 2 and m[1, 0] == 2 and m[1, 1] == 3
    assert make_matrix([5.0]).shape == (1, 1)


@pytest.mark.parametrize("hf,expected", [(3.015, 122), (3.0, 92)])
def test_lattice_neighbour_counts(oracle, hf, expected):
    # integer lattice (spacing 1): d^2 is exact, the strict d^2 < h^2 of
    # peri.jl:545 excludes |v|^2 = 9 for h = 3
    assert integer_vectors_below(hf * hf) == expected
    x, _ = lattice.cuboid(9, 9, 9, 1.0, centered=False)
    fam, intact = oracle.cal_family(x, hf, 200)
    counts = intact.sum(axis=0)
    centre = 4 + 9 * (4 + 9 * 4)
    assert counts[centre] == expected
    assert fam.shape[0] == counts.max() + 1  # trimmed to max count + 1 rows
    # descending, zero padded, symmetric
    for i in range(x.shape[1]):
        col = fam[:, i]
        nz = col[col > 0]
        assert np.all(np.diff(nz) < 0) and np.all(col[len(nz):] == 0)
    pairs = {(i, j - 1) for i in range(x.shape[1]) for j in fam[:, i] if j > 0}
    assert all((j, i) in pairs for i, j in pairs)


def test_family_overflow_raises(oracle):
    x, _ = lattice.cuboid(7, 7, 7, 1.0)
    with pytest.raises(IndexError):
        oracle.cal_family(x, 3.015, 122)  # needs max_neigh > 122
    oracle.cal_family(x, 3.015, 123)


def test_homogeneous_stretch_lps_dilatation(oracle):
    k = 1.002
    mat = lattice_block(7, 1.0e-3, 3.015, kind="lps", stretch=k)
    env = oracle.OracleEnv([mat], [], [], 1e-9)
    env.update_acc()
    th = env.blocks[0].theta
    # theta_i = 3/m_i sum |xi| (k-1)|xi| V_j = 3(k-1)  (peri.jl:168, 349)
    assert np.allclose(th, 3 * (k - 1), rtol=1e-9, atol=0)


def test_homogeneous_stretch_pmb_interior_zero_and_breaks(oracle):
    cs = 0.01
    for k, expect_broken in ((1 + 0.5 * cs, False), (1 + 1.5 * cs, True)):
        mat = lattice_block(9, 1.0e-3, 3.015, kind="pmb", stretch=k, cs=cs)
        env = oracle.OracleEnv([mat], [], [], 1e-9)
        env.update_acc()
        B = env.blocks[0]
        n_bonds = int((B.family > 0).sum())
        if expect_broken:
            assert B.intact.sum() == 0 and np.all(env.f == 0)
            assert np.all(env.damage() == 1.0)
        else:
            assert B.intact.sum() == n_bonds
            centre = 4 + 9 * (4 + 9 * 4)
            scale = np.abs(env.f).max()
            assert np.abs(env.f[:, centre]).max() <= 1e-9 * scale
            assert np.all(env.damage() == 0.0)


def test_rigid_translation_is_gated(oracle):
    mat = lattice_block(6, 1.0e-3, 3.015)
    mat.general.y[:] = mat.general.x + np.array([[1e-4], [-2e-4], [3e-4]])
    mat.general.deformed[0] = True  # y0 != x, but a rigid translate
    env = oracle.OracleEnv([mat], [], [], 1e-9)
    env.blocks[0].deformed = False
    env.update_acc()
    assert np.all(env.f == 0.0) and env.blocks[0].deformed is False


def test_momentum_conservation(oracle):
    w = configs.pmb_cube(n=8, spacing=1e-3, jitter=1e-5)
    env = oracle.OracleEnv(w["materials"], [], [], w["dt"])
    for _ in range(5):
        env.vv_step()
    mf = env.mass * env.f
    assert np.abs(mf.sum(axis=1)).max() <= 1e-9 * np.abs(mf).sum()


def pmb_energy(env):
    """Kinetic plus bond energy of a bond-based block.  The reference's
    per-bond term (t = c s, bond_based.jl:195-197; f_i += t/(2|Y|) Y V_j /
    rho_i from each of the bond's two visits, general_material.jl:340-360)
    is the force of the pair potential phi = c |xi| s^2 V_i V_j / 2, so
    velocity-Verlet must conserve sum m v^2 / 2 + sum over intact bonds of
    phi to O(dt^2)."""
    B = env.blocks[0]
    fam = B.family
    i = np.broadcast_to(np.arange(B.n), fam.shape)[fam > 0]
    j = fam[fam > 0] - 1
    xi = B.x[:, j] - B.x[:, i]
    Y = env.y[:, j] - env.y[:, i]
    lx = np.sqrt((xi * xi).sum(axis=0))
    s = (np.sqrt((Y * Y).sum(axis=0)) - lx) / lx
    live = B.intact[fam > 0] > 0
    phi = 0.5 * B.c[0, 0] * lx * s * s * B.vol[i] * B.vol[j]
    bond = 0.5 * phi[live].sum()  # every bond is listed in both families
    kinetic = 0.5 * (env.mass * (env.v * env.v).sum(axis=0)).sum()
    return kinetic, bond


def test_pmb_energy_is_conserved(oracle):
    w = configs.pmb_cube(n=8, spacing=1e-3, jitter=1e-5, peak=2.0, sigma=2e-3, cs=1.0)
    env = oracle.OracleEnv(w["materials"], [], [], w["dt"])
    env.update_acc()
    k0, b0 = pmb_energy(env)
    assert b0 == 0.0 and k0 > 0.0
    energies = []
    for _ in range(300):
        env.vv_step()
        energies.append(pmb_energy(env))
    assert env.blocks[0].intact.sum() == (env.blocks[0].family > 0).sum()  # nothing broke
    total = np.array([k + b for k, b in energies])
    # the pulse's energy has moved into the bonds, and the sum has stayed put
    assert max(b for _, b in energies) > 0.2 * k0
    assert np.abs(total - k0).max() <= 1e-4 * k0, np.abs(total - k0).max() / k0


def lps_energy(env):
    """Kinetic plus strain energy of a state-based block: the linear
    peridynamic solid's W_i = K theta_i^2 / 2 + 15 G / (2 m_i) sum_j
    omega (e - theta_i |xi| / 3)^2 V_j with omega = 1/|xi|, m_i = sum_j
    |xi| V_j (peri.jl:342-354) and theta_i = 3/m_i sum_j e V_j
    (peri.jl:155-172), computed here from the current positions.  Its
    gradient is the reference's bond term t = (3K - 5G)(theta_i/m_i +
    theta_j/m_j) omega |xi| + 15 G e omega (1/m_i + 1/m_j)
    (ordinary_state_based.jl:176-187)."""
    B = env.blocks[0]
    fam = B.family
    i = np.broadcast_to(np.arange(B.n), fam.shape)[fam > 0]
    j = fam[fam > 0] - 1
    xi = B.x[:, j] - B.x[:, i]
    Y = env.y[:, j] - env.y[:, i]
    lx = np.sqrt((xi * xi).sum(axis=0))
    e = np.sqrt((Y * Y).sum(axis=0)) - lx
    live = B.intact[fam > 0] > 0
    il, vl = i[live], B.vol[j[live]]
    m = np.zeros(B.n)
    np.add.at(m, il, lx[live] * vl)
    theta = np.zeros(B.n)
    np.add.at(theta, il, e[live] * vl)
    theta *= 3.0 / m
    ed = e[live] - theta[il] * lx[live] / 3.0
    dev = np.zeros(B.n)
    np.add.at(dev, il, ed * ed / lx[live] * vl)
    K, G = B.K[0, 0], B.G[0, 0]
    strain = (B.vol * (0.5 * K * theta * theta + 7.5 * G / m * dev)).sum()
    kinetic = 0.5 * (env.mass * (env.v * env.v).sum(axis=0)).sum()
    return kinetic, strain


def test_lps_energy_is_conserved(oracle):
    x, vol = lattice.cuboid(8, 8, 8, 1.0e-3, jitter=1.0e-5, seed=3)
    gen = GeneralMaterial(x.copy(order="F"), lattice.gaussian_pulse(x, 2.0, 2.0e-3), x, vol,
                          np.ones(x.shape[1], dtype=np.int64), 3.015e-3, max_neigh=200)
    mat = PeridynamicsMaterial(gen, OrdinaryStateBasedSpecific([14.9e9], [9.0e9], [1.0], [2200.0]))
    env = oracle.OracleEnv([mat], [], [], 1.0e-8)
    env.update_acc()
    k0, s0 = lps_energy(env)
    assert s0 == 0.0 and k0 > 0.0
    energies = []
    for _ in range(300):
        env.vv_step()
        energies.append(lps_energy(env))
    assert env.blocks[0].intact.sum() == (env.blocks[0].family > 0).sum()  # nothing broke
    total = np.array([k + s for k, s in energies])
    assert max(s for _, s in energies) > 0.2 * k0
    assert np.abs(total - k0).max() <= 1e-4 * k0, np.abs(total - k0).max() / k0


def test_contact12_energy_is_conserved(oracle):
    """Two bond-based cubes pressed together across a 0.9-spacing gap with
    nonlinear contact (exponent p = 2, stiffness 15 c).  The contact term
    (nonlinearspring.jl:124-145: K ((d - r)/d)^p / (r + 1e-10) dr, applied
    as F V2_j / rho1_i and -F V1_i / rho2_j, contacts.jl:210-247) is the
    force of the pair potential V1_i V2_j K d/(p+1) (1 - r/d)^(p+1) for
    r < d (the 1e-10 shifts it by ~1e-7 relative), so kinetic + bond +
    contact energy must stay put while the overlap pushes the cubes apart.
    Neighbours are rebuilt every step, and max_neighs exceeds the partner
    block's size, so every pair closer than d is listed."""
    sp, hf, K, rho = 1.0e-3, 3.015, 14.9e9, 2200.0

    def cube(origin, vx, t):
        x, vol = lattice.cuboid(5, 5, 5, sp, origin=origin, jitter=1e-5, seed=t + 2)
        v = np.zeros_like(x, order="F")
        v[0] = vx
        gen = GeneralMaterial(x.copy(order="F"), v, x, vol, np.full(x.shape[1], t, dtype=np.int64), hf * sp,
                              max_neigh=200)
        return PeridynamicsMaterial(gen, BondBasedSpecific([K], [1.0], [rho]), name=f"cube{t}")

    m1, m2 = cube((0.0, 0.0, 0.0), 5.0, 1), cube((4.9 * sp, 0.0, 0.0), -5.0, 2)
    c = 18 * K / math.pi / julia_pow_int(hf * sp, 4)
    con = NonLinearSpringContactModel(2.0, 15 * c, m1, m2, distanceX=3.0, max_neighs=200)
    env = oracle.OracleEnv([m1, m2], [con], [], 1e-8)
    d, p, Kc = con.equi_dist, 2.0, 15 * c

    def energy():
        kinetic = 0.5 * (env.mass * (env.v * env.v).sum(axis=0)).sum()
        bond = 0.0
        for B in env.blocks:
            fam = B.family
            i = np.broadcast_to(np.arange(B.n), fam.shape)[fam > 0]
            j = fam[fam > 0] - 1
            y = env.y[:, B.off:B.off + B.n]
            xi, Y = B.x[:, j] - B.x[:, i], y[:, j] - y[:, i]
            lx = np.sqrt((xi * xi).sum(axis=0))
            s = (np.sqrt((Y * Y).sum(axis=0)) - lx) / lx
            live = B.intact[fam > 0] > 0
            bond += 0.25 * (B.c[0, 0] * lx * s * s * B.vol[i] * B.vol[j])[live].sum()
        B1, B2 = env.blocks
        y1, y2 = env.y[:, B1.off:B1.off + B1.n], env.y[:, B2.off:B2.off + B2.n]
        r = np.sqrt(((y1[:, :, None] - y2[:, None, :]) ** 2).sum(axis=0))
        w = np.clip(1.0 - r / d, 0.0, None)
        contact = (B1.vol[:, None] * B2.vol[None, :] * Kc * d / (p + 1) * w ** (p + 1)).sum()
        return kinetic, bond, contact

    env.update_neighs()
    env.update_acc()
    k0, b0, c0 = energy()
    assert c0 > 10 * k0  # the cubes start overlapped by 0.1 d
    e0 = k0 + b0 + c0
    energies = []
    for _ in range(600):
        env.update_neighs()
        env.vv_step()
        energies.append(energy())
    total = np.array([sum(e) for e in energies])
    assert energies[-1][2] == 0.0 and energies[-1][0] > 0.5 * e0  # pushed apart: contact energy back in motion
    assert np.abs(total - e0).max() <= 1e-4 * e0, np.abs(total - e0).max() / e0


@pytest.mark.parametrize("kind", ["pmb", "lps"])
def test_gather_order_reproduces_serial_loop(oracle, kind):
    """The GPU's per-particle A/B/C gather equals the reference's serial
    scatter bit for bit, including the set of bonds broken."""
    rng = np.random.default_rng(7)
    mat = lattice_block(6, 1.0e-3, 3.015, kind=kind, jitter=2e-5, cs=0.002)
    env = oracle.OracleEnv([mat], [], [], 1e-9)
    B = env.blocks[0]
    env.y[:] = B.x + rng.normal(0.0, 1.5e-6, size=B.x.shape)
    intact_before = B.intact.copy()
    env.update_acc()
    assert 0 < (intact_before.sum() - B.intact.sum()) < intact_before.sum()  # some, not all, broke
    spc = mat.specific
    theta = None
    if kind == "lps":
        theta = gather_order.gather_theta(B.x, env.y, B.family, intact_before.astype(bool), B.vol, B.m)
        assert np.array_equal(theta, B.theta)
    f, intact_after = gather_order.gather_force(
        0 if kind == "pmb" else 1, B.x, env.y, B.family, intact_before.astype(bool), B.type_rel, B.cs, B.density,
        B.vol, B.c, m=B.m, theta=theta, K=getattr(spc, "bulk_modulus", None), G=getattr(spc, "shear_modulus", None))
    assert np.array_equal(f, env.f)
    assert np.array_equal(intact_after, B.intact.astype(bool))


def test_threaded_oracle_matches_serial(oracle):
    w1 = configs.pmb_cube(n=8, spacing=1e-3, jitter=1e-5)
    e1 = oracle.OracleEnv(w1["materials"], [], [], w1["dt"], nthreads=1)
    e4 = oracle.OracleEnv(w1["materials"], [], [], w1["dt"], nthreads=4)
    for _ in range(3):
        e1.vv_step()
        e4.vv_step()
    assert np.allclose(e1.y, e4.y, rtol=1e-13, atol=0)
    assert np.array_equal(e1.blocks[0].intact, e4.blocks[0].intact)


def test_contact11_merge_walk_only_matches_first_member(oracle):
    """The reference's merge walk (contacts.jl:539-573) scans the family
    column from its largest entry, so only that entry can become a contact
    neighbour -- the closed form the GPU kernel uses."""
    rng = np.random.default_rng(3)
    x, vol = lattice.cuboid(7, 7, 4, 1.0, jitter=0.05, seed=5)
    fam, intact = oracle.cal_family(x, 3.015, 200)
    intact = np.asfortranarray(intact & (rng.random(intact.shape) > 0.3), dtype=np.uint8)
    y = np.asfortranarray(x + rng.normal(0, 0.1, size=x.shape))
    n = x.shape[1]
    rows = 50
    for equi in (1.0, 1.5, 3.5):
        nb = np.zeros((rows, n), dtype=np.int64, order="F")
        oracle.lib().or_contact11_neighs(n, oracle._d(y), fam.shape[0], oracle._i(fam), oracle._u(intact), 5.0, equi,
                                         30, rows, oracle._i(nb))
        assert np.all(nb[1:] == 0)
        for i in range(n):
            q = fam[0, i]
            expect = 0
            if q > 0 and not intact[0, i]:
                d = y[:, i] - y[:, q - 1]
                if d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < equi * equi:
                    expect = q
            assert nb[0, i] == expect


def test_contact11_ordered_search_bruteforce(oracle):
    """The ordered self-contact search lists every broken-bond family member
    in an adjacent get_cells cell and within equi_dist, in family order; its
    first entry agrees with the reference's merge walk wherever that finds
    one."""
    rng = np.random.default_rng(4)
    x, vol = lattice.cuboid(7, 7, 4, 1.0, jitter=0.05, seed=5)
    fam, intact = oracle.cal_family(x, 3.015, 200)
    intact = np.asfortranarray(intact & (rng.random(intact.shape) > 0.3), dtype=np.uint8)
    y = np.asfortranarray(x + rng.normal(0, 0.1, size=x.shape))
    n = x.shape[1]
    h, max_part, rows = 2.5, 30, 12
    mn, mx = y.min(axis=1), y.max(axis=1)
    N = np.clip(np.floor((mx - mn) / h), 1, max_part)
    cell = np.clip(np.floor((y - mn[:, None]) / h), 1, max_part)
    assert np.all(cell <= N[:, None])
    for equi in (1.0, 1.5, 3.5):
        ref = np.zeros((rows, n), dtype=np.int64, order="F")
        nb = np.zeros((rows, n), dtype=np.int64, order="F")
        args = (n, oracle._d(y), fam.shape[0], oracle._i(fam), oracle._u(intact), h, equi, max_part, rows)
        oracle.lib().or_contact11_neighs(*args, oracle._i(ref))
        oracle.lib().or_contact11_neighs_ordered(*args, oracle._i(nb))
        longest = 0
        for i in range(n):
            expect = []
            for k in range(fam.shape[0]):
                j = fam[k, i] - 1
                if j < 0 or intact[k, i] or np.any(np.abs(cell[:, i] - cell[:, j]) > 1):
                    continue
                d = y[:, i] - y[:, j]
                if (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2] < equi * equi:
                    expect.append(j + 1)
            expect = expect[:rows]
            longest = max(longest, len(expect))
            assert list(nb[:len(expect), i]) == expect
            assert np.all(nb[len(expect):, i] == 0)
            if ref[0, i]:
                assert nb[0, i] == ref[0, i]
        if equi > 3:
            assert longest > 1


def test_contact12_neighs_bruteforce(oracle):
    rng = np.random.default_rng(11)
    x1 = np.asfortranarray(rng.uniform(0, 4, size=(3, 300)))
    x2 = np.asfortranarray(rng.uniform(2, 6, size=(3, 400)))
    dist, rows = 0.9, 7
    nb = np.zeros((rows, 300), dtype=np.int64, order="F")
    oracle.lib().or_contact12_neighs(300, oracle._d(x1), 400, oracle._d(x2), dist, rows, oracle._i(nb))
    lo = np.maximum(x1.min(axis=1) - dist, x2.min(axis=1) - dist)
    hi = np.minimum(x1.max(axis=1) + dist, x2.max(axis=1) + dist)
    in2 = np.all((x2 > lo[:, None]) & (x2 < hi[:, None]), axis=0)
    for i in range(300):
        if not np.all((x1[:, i] > lo) & (x1[:, i] < hi)):
            assert np.all(nb[:, i] == 0)
            continue
        d = x1[:, i:i + 1] - x2
        d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
        cand = np.nonzero(in2 & (d2 < dist * dist))[0] + 1
        expect = np.zeros(rows, dtype=np.int64)
        top = np.sort(cand)[::-1][:rows]
        expect[: top.size] = top
        assert np.array_equal(nb[:, i], expect)


def test_fix_and_tofro_bcs_known_answers(oracle):
    """FixBC.jl:46-65: the masked coordinates stay at their t0 snapshot with
    zero velocity.  ToFroBC.jl:51-111 within velocity_verlet.jl:57-89: each
    step moves the masked coordinates by dt * direction * rate from where
    the previous step left them and sets v = direction * rate; check! after
    the step flips the direction when time_step > applyafter and time_step
    % freq == 0 (time_step counted before its increment).  Unconstrained
    coordinates (dims false) move freely."""
    from peridyn_b200 import FixBC, ToFroBC

    mat = lattice_block(6, 1.0e-3, 3.015, kind="lps")
    x = mat.general.x
    left, right = x[0] < x[0].min() + 1.5e-3, x[0] > x[0].max() - 1.5e-3
    rate = np.array([2.0, 0.3, 0.0])
    bcs = [FixBC(left), ToFroBC(right, rate, 4, dims=(True, True, False), applyafter=2)]
    env = oracle.OracleEnv([mat], [], bcs, 1.0e-8)
    env.apply_bc_at0()
    y0 = env.y.copy()
    il, ir = np.nonzero(left)[0], np.nonzero(right)[0]
    direction, moved = 1, np.zeros(3)
    for ts in range(14):
        env.vv_step()
        moved += env.dt * direction * rate
        assert np.array_equal(env.y[:, il], y0[:, il]) and np.all(env.v[:, il] == 0.0)
        for d in (0, 1):
            assert np.allclose(env.y[d, ir], y0[d, ir] + moved[d], rtol=0, atol=1e-15)
            assert np.all(env.v[d, ir] == direction * rate[d])
        if ts > 2 and ts % 4 == 0:
            direction = -direction
    # flips after steps 4, 8 and 12: the run ends moving in the negative direction
    assert direction == -1 and np.all(env.v[0, ir] == -rate[0])
    assert not np.array_equal(env.y[2, ir], y0[2, ir])  # z is not constrained and has moved


def test_scaling_bcs_known_answers(oracle):
    # DeltaScaleBC.jl:52-55: y = (last - fix) * (1 + scale*dt*time_step) + fix
    from tests.cases import bar_with_bcs

    w = bar_with_bcs("delta")
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"])
    ora.apply_bc_at0()
    bc = ora.bcs[1]
    last = bc.last.copy()
    idx = np.nonzero(bc.mask)[0]
    for ts in range(3):
        ora.vv_step()  # position BC applied with time_step = ts
        g = 1.0 + (bc.scale * ora.dt) * float(ts)
        want = (last - bc.fixpoint[:, None]) * g[:, None] + bc.fixpoint[:, None]
        assert np.array_equal(ora.y[:, idx], want)
        assert np.all(ora.v[:, idx] == 0.0)
    # ScaleFixWaitBC.jl:63-68: check! at time_step 0 scales the scalebool set
    w = bar_with_bcs("scalefixwait")
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"])
    ora.apply_bc_at0()
    bc = ora.bcs[1]
    y0 = ora.y.copy()
    ora.vv_step()
    s = np.nonzero(bc.smask & ~ora.bcs[0].mask)[0]
    g = np.sqrt(1.0 + 2.0 * bc.scale[0] * ora.dt)
    assert g > 1.0
    # x of the scaled particles moved away from the fix point by the factor
    ratio = (ora.y[0, s] - bc.fixpoint[0]) / (y0[0, s] - bc.fixpoint[0])
    assert np.all(ratio > 1.0 + 0.5 * (g - 1.0))
    assert np.array_equal(bc.last, ora.y[:, bc.mask])


def test_container_bc_zeroes_escaping_velocities(oracle):
    from tests.cases import bar_with_bcs

    w = bar_with_bcs("container")
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"])
    ora.apply_bc_at0()
    bc = ora.bcs[1]
    idx = np.nonzero(bc.mask)[0]
    outside_seen = False
    for _ in range(40):
        ora.vv_step()
        yb = ora.y[:, idx]
        out = np.any((yb < bc.limits[:, :1]) | (yb > bc.limits[:, 1:]), axis=0)
        assert np.all(ora.v[:, idx[out]] == 0.0)
        outside_seen |= bool(out.any())
    assert outside_seen


def test_elasto_plastic_elastic_limit_is_lps(oracle):
    # With a yield stress too high to be reached, C = sqrt(2 psi / td_norm2)
    # stays > 1 and t = 3K |xi| tw + 15G (a + b) ed, which is the LPS law
    # (ordinary_state_based.jl:176-187) rearranged: same forces to rounding.
    import peridyn_b200 as pb
    from tests.cases import ep_cube

    w = ep_cube(1e30, n=8)
    gen = w["materials"][0].general
    lps = pb.PeridynamicsMaterial(gen, pb.OrdinaryStateBasedSpecific([46.7e9], [28.0e9], [0.02], [2700.0]))
    a = oracle.OracleEnv(w["materials"], [], [], w["dt"])
    b = oracle.OracleEnv([lps], [], [], w["dt"])
    for _ in range(25):
        a.vv_step()
        b.vv_step()
    assert np.all(a.blocks[0].edp == 0.0)
    assert np.linalg.norm(a.y - b.y) <= 1e-12 * np.linalg.norm(b.y)
    assert np.linalg.norm(a.f - b.f) <= 1e-9 * np.linalg.norm(b.f)


def test_elasto_plastic_yields(oracle):
    from tests.cases import ep_cube

    w = ep_cube(5e6, n=8)
    a = oracle.OracleEnv(w["materials"], [], [], w["dt"])
    for _ in range(25):
        a.vv_step()
    B = a.blocks[0]
    assert np.abs(B.edp).max() > 0.0
    assert np.all(B.edp[B.family == 0] == 0.0)
