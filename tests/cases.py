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
