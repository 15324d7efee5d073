"""Shared test workloads."""
import numpy as np

import peridyn_b200 as pb
from peridyn_b200 import lattice


def random_cloud():
    # disordered points: neighbour offsets differ from lane to lane, so the
    # slices keep explicit indices
    rng = np.random.default_rng(21)
    n, L = 1500, 12e-3
    x = np.asfortranarray(rng.uniform(0.0, L, size=(3, n)))
    vol = np.full(n, L ** 3 / n)
    gen = pb.GeneralMaterial(x.copy(order="F"), lattice.gaussian_pulse(x, 5.0, 3e-3), x, vol,
                             np.ones(n, dtype=np.int64), 2.6e-3, max_neigh=300)
    mat = pb.PeridynamicsMaterial(gen, pb.OrdinaryStateBasedSpecific([20e9], [9e9], [0.004], [2000.0]))
    return {"materials": [mat], "contacts": [], "bcs": [], "dt": 2e-8, "steps": 20}


def bar_with_bcs(kind, nx=20, ny=6, nz=6, steps=60):
    """LPS bar with one of the scaling / container boundary conditions
    beside a FixBC on the x = min layers."""
    from peridyn_b200 import configs

    w = configs.lps_bar(nx=nx, ny=ny, nz=nz, steps=steps)
    mat = w["materials"][0]
    x = mat.general.x
    h = mat.general.horizon
    xmin, xmax = x[0].min(), x[0].max()
    fix = pb.FixBC(x[0] < xmin + h)
    right = x[0] > xmax - h
    cen = x.mean(axis=1)
    if kind == "delta":
        bc = pb.DeltaScaleBC(right, [2.0e3, 500.0, 0.0], [xmin, cen[1], cen[2]])
    elif kind == "scalefixwait":
        bc = pb.ScaleFixWaitBC(right, [3.0e3, 0.0, 0.0], [xmin, cen[1], cen[2]], 10, x[0] > cen[0])
    else:
        # the pull drives the right end out of the box; its velocity is zeroed there
        lim = np.array([[xmin - h, xmax + 2.0e-7], [x[1].min() - h, x[1].max() + h], [x[2].min() - h, x[2].max() + h]])
        mat.general.velocity[0] = np.where(right, 2.0, 0.0)
        bc = pb.ContainerBC(x[0] > cen[0], limits=lim)
    w["bcs"] = [fix, bc]
    return w


def ep_cube(sigma_y, n=10, peak=60.0, cs=0.02, seed=7, ntypes=1):
    """Elasto-plastic (Von Mises) cube with the pmb_cube pulse; a second
    type on the x > mean half when ntypes == 2."""
    x, vol = lattice.cuboid(n, n - 1, n - 2, 1.0e-3, jitter=1.0e-5, seed=seed)
    t = np.ones(x.shape[1], dtype=np.int64)
    if ntypes == 2:
        t = np.where(x[0] < x[0].mean(), 1, 2).astype(np.int64)
    gen = pb.GeneralMaterial(x.copy(order="F"), lattice.gaussian_pulse(x, peak, 3.0e-3), x, vol, t, 3.015e-3,
                             max_neigh=200)
    # per type-pair values in make_matrix order (n(n+1)/2 entries for n types)
    npairs = ntypes * (ntypes + 1) // 2
    K = [46.7e9, 43.0e9, 40.0e9][:npairs]
    G = [28.0e9, 26.0e9, 25.0e9][:npairs]
    sy = [sigma_y, 1.5 * sigma_y, 2.0 * sigma_y][:npairs]
    spc = pb.ElastoPlasticSolidSpecific(K, G, [cs] * npairs, [2700.0, 2500.0][:ntypes], sy)
    mat = pb.PeridynamicsMaterial(gen, spc, name="ep_cube")
    return {"materials": [mat], "contacts": [], "bcs": [], "dt": 2.0e-8, "steps": 60}


def self_contact_block(oracle, ordered=False, max_neighs=20, seed=8):
    """A block with a random third of its bonds broken (symmetrically),
    compressed to 0.7x so broken pairs come within the contact distance of a
    linear-spring self contact.  Returns the workload and the families
    (computed by the oracle) both sides are given."""
    x, vol = lattice.cuboid(8, 8, 6, 1e-3, jitter=3e-5, seed=2)
    fam, intact = oracle.cal_family(x, 3.015e-3, 200)
    rng = np.random.default_rng(seed)
    n = x.shape[1]
    brk = set()
    for i in range(n):
        for k in range(fam.shape[0]):
            j = fam[k, i]
            if j > 0 and j - 1 > i and rng.random() < 0.35:
                brk.add((i, j - 1))
    intact = intact.copy()
    for i in range(n):
        for k in range(fam.shape[0]):
            j = fam[k, i] - 1
            if j >= 0 and ((i, j) in brk or (j, i) in brk):
                intact[k, i] = False
    y = np.asfortranarray(0.7 * x + rng.normal(0, 5e-5, size=x.shape))
    gen = pb.GeneralMaterial(y, np.zeros_like(x, order="F"), x, vol, np.ones(n, dtype=np.int64), 3.015e-3,
                             max_neigh=200)
    mat = pb.PeridynamicsMaterial(gen, pb.BondBasedSpecific([10e9], [0.5], [2000.0]))
    cm = pb.LinearSpringContactModel(1e18, mat, distanceX=5, max_neighs=max_neighs, ordered=ordered)
    return {"materials": [mat], "contacts": [cm], "bcs": [], "dt": 1e-9}, [(fam, intact)]
