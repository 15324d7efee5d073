"""Edge cases of the particle and bond layout against the oracle, in all
three precisions, in one environment of four blocks:

  * a block of one particle (no family at all);
  * a block of two particles (one bond each way);
  * a 33-particle state-based plate (a slice of 32 and a slice of one
    particle padded by 31 lanes);
  * a cube with one particle far from the rest (an empty family inside a
    block whose other families are full: damage 0/0 = NaN, as cal_damage
    gives it, peri.jl:587-594).

Tolerances: serial FP64 bit-identical (y, v, f, damage with NaN in the
same places); one-pass FP64 displacement and velocity rel-L2 <= 1e-10;
FP32C <= 1e-4."""
import numpy as np
import pytest

import peridyn_b200 as pb
from peridyn_b200 import lattice

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32c": 1e-4}


def _block(x, kind, type_id, seed):
    n = x.shape[1]
    rng = np.random.default_rng(seed)
    v = np.asfortranarray(rng.uniform(-5.0, 5.0, size=(3, n)))
    vol = np.full(n, 1.0e-9)
    gen = pb.GeneralMaterial(np.asfortranarray(x.copy()), v, np.asfortranarray(x), vol,
                             np.full(n, type_id, dtype=np.int64), 3.015e-3, max_neigh=200)
    if kind == "pmb":
        spc = pb.BondBasedSpecific([14.9e9], [0.005], [2200.0])
    else:
        spc = pb.OrdinaryStateBasedSpecific([20e9], [9e9], [0.004], [2000.0])
    return pb.PeridynamicsMaterial(gen, spc, name=f"edge{type_id}")


def _workload():
    one = np.zeros((3, 1))
    two = np.array([[0.0, 1.0e-3], [0.0, 0.0], [0.0, 0.0]])
    plate, _ = lattice.cuboid(11, 3, 1, 1.0e-3, jitter=1.0e-5, seed=3)
    cube, _ = lattice.cuboid(5, 5, 5, 1.0e-3, jitter=1.0e-5, seed=4)
    # 50 mm from the rest, far outside the 3 mm horizon (and near enough
    # that the reference's absolute-position update, y += dt v, keeps the
    # displacement's digits: at 1 m its rounding alone would exceed 1e-10)
    cube = np.hstack([cube, [[0.05], [0.05], [0.05]]])
    mats = [_block(one, "pmb", 1, 1), _block(two, "pmb", 2, 2), _block(plate, "lps", 3, 3),
            _block(cube, "pmb", 4, 4)]
    return {"materials": mats, "contacts": [], "bcs": [], "dt": 1.0e-8}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("precision", ["fp64_serial", "fp64", "fp32c"])
def test_tiny_ragged_and_empty_families(oracle, precision):
    w = _workload()
    nsteps = 60
    env = pb.Env(1, w["materials"], w["contacts"], w["bcs"], w["dt"], precision=precision)
    ora = oracle.OracleEnv(w["materials"], w["contacts"], w["bcs"], w["dt"])
    assert env.N == 1 + 2 + 33 + 126
    assert np.array_equal(np.asarray(env.intact0), ora.intact0)
    assert int(ora.intact0[0]) == 0 and int(ora.intact0[-1]) == 0 and int(ora.intact0[1]) == 1
    for _ in range(nsteps):
        ora.vv_step()
    pb.velocity_verlet_step(env, nsteps=nsteps)
    y, v, f, _ = env.get_state()
    d = pb.cal_damage(env)
    dref = ora.damage()
    assert np.array_equal(np.isnan(d), np.isnan(dref))
    assert np.isnan(d[0]) and np.isnan(d[-1])
    x = np.hstack([B.x for B in ora.blocks])
    if precision == "fp64_serial":
        assert np.array_equal(y, ora.y)
        assert np.array_equal(v, ora.v)
        assert np.array_equal(d, dref, equal_nan=True)
    else:
        assert _rel(y - x, ora.y - x) <= TOL[precision]
        assert _rel(v, ora.v) <= TOL[precision]
        ok = ~np.isnan(dref)
        assert np.array_equal(d[ok], dref[ok])
    # the lone particles move ballistically
    v_one = w["materials"][0].general.velocity[:, 0]
    v_far = w["materials"][3].general.velocity[:, -1]
    for p, v0 in ((0, v_one), (env.N - 1, v_far)):
        assert np.allclose(y[:, p], x[:, p] + nsteps * w["dt"] * v0, rtol=0, atol=1e-12)
    env.close()
