"""The runtime bond layout converted on the device (the default) against the
host conversion (PD_LAYOUT_HOST=1), on lattices, a disordered cloud, a
contact workload and a batch of specimens, in the stencil and the explicit
forms: the same layout statistics (slices, stencil slices, bond slots,
index entries, staged slices), the same families and intact flags in the
reference layout, and bit-identical trajectories in FP32C (the walks read
every array the conversion writes)."""
import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import configs
from tests.cases import random_cloud

pytestmark = pytest.mark.gpu

BUILDERS = {
    "pmb_cube": lambda: configs.pmb_cube(n=12, peak=40.0),
    "lps_bar": lambda: configs.lps_bar(nx=40, ny=10, nz=10),
    "cloud": random_cloud,
    "disk": lambda: configs.disk_impact(radius=3.0e-3, thickness=1.0e-3, spacing=2.5e-4, sphere_radius=1.0e-3,
                                        speed=300.0),
    "batched": lambda: configs.batched_cubes(nspec=8, edge_lo=12, edge_hi=20),
}


def _env(w, monkeypatch, host):
    if host:
        monkeypatch.setenv("PD_LAYOUT_HOST", "1")
    else:
        monkeypatch.delenv("PD_LAYOUT_HOST", raising=False)
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision="fp32c")
    monkeypatch.delenv("PD_LAYOUT_HOST", raising=False)
    return env


def _run(env, w, nsteps):
    if w["bcs"]:
        pb.apply_bc_at0(env, 0)
    if w["contacts"]:
        pb.update_neighs(env)
        pb.update_acc(env)
    pb.velocity_verlet_step(env, nsteps=nsteps)
    return env.get_state()


@pytest.mark.parametrize("layout", ["auto", "explicit"])
@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_device_layout_equals_host_layout(name, layout, monkeypatch):
    if layout == "explicit":
        monkeypatch.setenv("PD_FAMILY_LAYOUT", "explicit")
    else:
        monkeypatch.delenv("PD_FAMILY_LAYOUT", raising=False)
    w = BUILDERS[name]()
    eh = _env(w, monkeypatch, host=True)
    ed = _env(w, monkeypatch, host=False)
    assert eh.layout() == ed.layout()
    lay = ed.layout()
    # every bond is walked; no slice walks past its slot list
    assert ed.num_bonds() <= lay["walked_slots"] <= lay["slots"]
    if layout == "auto" and name != "cloud":
        assert ed.layout()["stencil_slices"] > 0
    for b in range(len(w["materials"])):
        fh, ih = eh._family(b)
        fd, idd = ed._family(b)
        assert np.array_equal(fh, fd) and np.array_equal(ih, idd)
    for a, b in zip(_run(eh, w, 40), _run(ed, w, 40)):
        assert np.array_equal(a, b)
    eh.close()
    ed.close()
