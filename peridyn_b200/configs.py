"""Workload builders: the benchmark specimens, generated synthetically.

Each builder returns a dict with ``materials``, ``contacts``, ``bcs``,
``dt`` and ``steps`` that can be handed to :func:`peridyn_b200.Env` (and to
the oracle).  Sizes are parameters so that tests can run scaled-down
versions of the same setups.
"""
import math

import numpy as np

from . import lattice
from .boundary_conditions import FixBC, MoveBC
from .contacts import NonLinearSpringContactModel
from .materials import (BondBasedSpecific, GeneralMaterial, OrdinaryStateBasedSpecific, PeridynamicsMaterial,
                        julia_pow_int)


def pmb_cube(n=20, spacing=1.0e-3, jitter=1.0e-5, seed=1, horizon_factor=3.015, rho=2200.0, K=14.9e9,
             cs=0.005, peak=10.0, sigma=3.0e-3, dt=1.0e-8, steps=1000, origin=(0.0, 0.0, 0.0), type_id=1,
             name="cube", dims=None):
    """Plain bond-based cube: n^3 lattice, Gaussian velocity pulse on the
    x=min face, no boundary conditions, no contact."""
    nx, ny, nz = dims if dims is not None else (n, n, n)
    x, vol = lattice.cuboid(nx, ny, nz, spacing, origin=origin, jitter=jitter, seed=seed)
    y = x.copy(order="F")
    v = lattice.gaussian_pulse(x, peak, sigma)
    t = np.full(x.shape[1], type_id, dtype=np.int64)
    gen = GeneralMaterial(y, v, x, vol, t, horizon_factor * spacing, max_neigh=200)
    spc = BondBasedSpecific([K], [cs], [rho])
    mat = PeridynamicsMaterial(gen, spc, name=name)
    return {"materials": [mat], "contacts": [], "bcs": [], "dt": dt, "steps": steps,
            "workload": f"pmb_cube_{nx}x{ny}x{nz}"}


def lps_bar(nx=100, ny=20, nz=20, spacing=5.0e-4, horizon_factor=3.0, E=70e9, nu=0.25, rho=2700.0, cs=0.01,
            pull=2.0, dt=5.0e-9, steps=5000):
    """Ordinary state-based tensile bar: exact lattice x = i*spacing, FixBC
    on x < x_min + horizon, MoveBC at +pull m/s on x > x_max - horizon."""
    x, vol = lattice.cuboid(nx, ny, nz, spacing, centered=False)
    y = x.copy(order="F")
    v = np.zeros_like(x, order="F")
    t = np.ones(x.shape[1], dtype=np.int64)
    horizon = horizon_factor * spacing
    gen = GeneralMaterial(y, v, x, vol, t, horizon, max_neigh=200)
    K = E / 3 / (1 - 2 * nu)
    G = E / 2 / (1 + nu)
    spc = OrdinaryStateBasedSpecific([K], [G], [cs], [rho])
    mat = PeridynamicsMaterial(gen, spc, name="bar")
    xmin, xmax = x[0].min(), x[0].max()
    bc1 = FixBC(x[0] < xmin + horizon)
    bc2 = MoveBC(x[0] > xmax - horizon, [pull, 0.0, 0.0])
    return {"materials": [mat], "contacts": [], "bcs": [bc1, bc2], "dt": dt, "steps": steps,
            "workload": f"lps_bar_{nx}x{ny}x{nz}"}


def batched_cubes(nspec=256, seed=4, edge_lo=12, edge_hi=32, spacing=1.0e-3, steps=2000, dt=1.0e-8,
                  cs_lo=0.002, cs_hi=0.01, v_lo=5.0, v_hi=50.0, cubes=False):
    """Independent PMB cuboids of uneven size (edges uniform over
    edge_lo..edge_hi per axis), critical stretch U(cs_lo, cs_hi), pulse peak
    U(v_lo, v_hi).  Specimens are separate blocks (type id = block index).
    cubes=True: one drawn edge per specimen (cubes of edge_lo^3 to
    edge_hi^3 particles) instead of one per axis."""
    u = lattice.uniform(seed, 5 * nspec)
    mats = []
    for s in range(nspec):
        e = [edge_lo + int(u[5 * s + (0 if cubes else d)] * (edge_hi - edge_lo + 1)) for d in range(3)]
        cs = cs_lo + (cs_hi - cs_lo) * u[5 * s + 3]
        peak = v_lo + (v_hi - v_lo) * u[5 * s + 4]
        origin = (s * 40 * spacing, 0.0, 0.0)
        w = pmb_cube(dims=e, spacing=spacing, seed=seed * 100003 + s, cs=cs, peak=peak, origin=origin,
                     type_id=s + 1, name=f"specimen{s}", dt=dt, steps=steps)
        mats.extend(w["materials"])
    return {"materials": mats, "contacts": [], "bcs": [], "dt": dt, "steps": steps,
            "workload": f"batched_{nspec}_pmb" + ("_cubes" if cubes else "")}


def disk_impact(radius=0.05, thickness=0.005, spacing=2.5e-4, sphere_radius=0.01, speed=100.0, cs=0.003,
                horizon_factor=3.015, rho=2200.0, K=14.9e9, stiff_factor=100.0, contact_factor=15.0, steps=10000,
                dt=None, gap=None):
    """Bond-based disk (axis z) hit along -z by a stiff bond-based sphere,
    nonlinear contact (exponent 2) of stiffness contact_factor * c with
    equilibrium distance = spacing and search distance = horizon.  ``gap``
    is the z clearance between the lowest projectile particle and the
    highest disk particle (default 0.9 spacing: inside the contact distance,
    so the impact starts at the first step)."""
    horizon = horizon_factor * spacing
    xd, vd = lattice.disk(radius, thickness, spacing)
    gap = 0.9 * spacing if gap is None else gap
    xs0, _ = lattice.sphere(sphere_radius, spacing, center=(0.0, 0.0, 0.0))
    zc = xd[2].max() + gap - xs0[2].min()
    xs, vs = lattice.sphere(sphere_radius, spacing, center=(0.0, 0.0, zc))
    gen_d = GeneralMaterial(xd.copy(order="F"), np.zeros_like(xd, order="F"), xd, vd,
                            np.full(xd.shape[1], 1, dtype=np.int64), horizon, max_neigh=200)
    vsph = np.zeros_like(xs, order="F")
    vsph[2] = -speed
    gen_s = GeneralMaterial(xs.copy(order="F"), vsph, xs, vs, np.full(xs.shape[1], 2, dtype=np.int64), horizon,
                            max_neigh=200)
    disk_m = PeridynamicsMaterial(gen_d, BondBasedSpecific([K], [cs], [rho]), name="disk")
    sph_m = PeridynamicsMaterial(gen_s, BondBasedSpecific([stiff_factor * K], [1.0], [rho]), name="projectile")
    c = 18 * K / math.pi / julia_pow_int(horizon, 4)
    contact = NonLinearSpringContactModel(2.0, contact_factor * c, sph_m, disk_m, distanceD=1.0,
                                          distanceX=horizon_factor, max_neighs=50)
    if dt is None:
        # PMB critical time step estimate sqrt(2 rho / sum_j c_stiff V_j / |xi|), halved
        nvol = spacing ** 3
        csph = stiff_factor * c
        kx = 0.0
        r = int(math.ceil(horizon_factor))
        for i in range(-r, r + 1):
            for j in range(-r, r + 1):
                for k in range(-r, r + 1):
                    d = math.sqrt(i * i + j * j + k * k) * spacing
                    if 0 < d < horizon:
                        kx += csph * nvol / d
        dt = 0.5 * math.sqrt(2 * rho / kx)
    return {"materials": [sph_m, disk_m], "contacts": [contact], "bcs": [], "dt": dt, "steps": steps,
            "workload": "disk_impact"}


def lps_cube(dims, spacing=1.0e-3, jitter=1.0e-5, seed=1, horizon_factor=3.015, E=70e9, nu=0.25, rho=2700.0,
             cs=0.01, peak=10.0, sigma=3.0e-3, dt=1.0e-8, steps=1000):
    """State-based (LPS) cuboid with the Gaussian pulse of pmb_cube."""
    nx, ny, nz = dims
    x, vol = lattice.cuboid(nx, ny, nz, spacing, jitter=jitter, seed=seed)
    gen = GeneralMaterial(x.copy(order="F"), lattice.gaussian_pulse(x, peak, sigma), x, vol,
                          np.ones(x.shape[1], dtype=np.int64), horizon_factor * spacing, max_neigh=200)
    K = E / 3 / (1 - 2 * nu)
    G = E / 2 / (1 + nu)
    mat = PeridynamicsMaterial(gen, OrdinaryStateBasedSpecific([K], [G], [cs], [rho]), name="lps_cube")
    return {"materials": [mat], "contacts": [], "bcs": [], "dt": dt, "steps": steps,
            "workload": f"lps_cube_{nx}x{ny}x{nz}"}


def serving_jobs(njobs, seed=5, rate=50.0, n_lo=5.0e3, n_hi=5.0e5, steps_lo=500, steps_hi=5000,
                 precision="fp32c"):
    """Mixed stream of PMB and state-based cube jobs: particle counts
    log-uniform over [n_lo, n_hi], steps uniform over steps_lo..steps_hi,
    critical stretch U(0.002, 0.01) and pulse peak U(5, 50) m/s as in
    batched_cubes; Poisson arrivals at ``rate`` jobs/s.  Returns (jobs,
    arrival times in s)."""
    u = lattice.uniform(seed, 6 * njobs)
    jobs, arrivals, t = [], [], 0.0
    for k in range(njobs):
        uk = u[6 * k:6 * k + 6]
        n = math.exp(math.log(n_lo) + (math.log(n_hi) - math.log(n_lo)) * uk[0])
        e = max(4, int(round(n ** (1.0 / 3.0))))
        nsteps = steps_lo + int(uk[1] * (steps_hi - steps_lo + 1))
        cs = 0.002 + 0.008 * uk[2]
        peak = 5.0 + 45.0 * uk[3]
        if uk[4] < 0.5:
            w = pmb_cube(dims=(e, e, e), cs=cs, peak=peak, seed=seed * 7919 + k, steps=nsteps)
        else:
            w = lps_cube((e, e, e), cs=cs, peak=peak, seed=seed * 7919 + k, steps=nsteps)
        w["nsteps"] = nsteps
        w["precision"] = precision
        jobs.append(w)
        t += -math.log(1.0 - uk[5]) / rate
        arrivals.append(t)
    return jobs, arrivals


def ep_bar(nx=100, ny=20, nz=20, yield_stress=2e6, steps=2000):
    """The lps_bar tensile bar (Fix + Move BCs) as an elasto-plastic (Von
    Mises) solid with the given yield stress."""
    from .materials import ElastoPlasticSolidSpecific

    w = lps_bar(nx=nx, ny=ny, nz=nz, steps=steps)
    mat = w["materials"][0]
    E, nu = 70e9, 0.25
    K = E / 3 / (1 - 2 * nu)
    G = E / 2 / (1 + nu)
    spc = ElastoPlasticSolidSpecific([K], [G], [0.01], [2700.0], [yield_stress])
    w["materials"] = [PeridynamicsMaterial(mat.general, spc, name="ep_bar")]
    w["workload"] = f"ep_bar_{nx}x{ny}x{nz}"
    return w
