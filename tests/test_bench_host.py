"""Host logic of bench.py: the algorithmic byte model behind the roofline
(4.125 B per intact directed bond and per bond sweep, 84 / 168 B per
particle, 8 B more for state-based blocks),
the compute roofline's arithmetic, the bounded CPU sample of the batched
workload and its cube-edge variant, and the serving sample's stream."""
import bench
from peridyn_b200 import configs


def test_step_bytes_model():
    # bond-based FP32C: 4.125 B per intact directed bond, 84 B per particle
    assert bench.step_bytes(1000, 10, "fp32c", False) == 4.125 * 1000 + 84 * 10
    # FP64: 168 B per particle
    assert bench.step_bytes(1000, 10, "fp64", False) == 4.125 * 1000 + 168 * 10
    # state-based: two bond sweeps and the dilatation (8 B) per particle
    assert bench.step_bytes(1000, 10, "fp32c", True) == 2 * 4.125 * 1000 + 92 * 10
    # the 256-specimen batched workload: 290,639,420 bonds, 2,815,119 particles, 1.435 GB per step
    assert abs(bench.step_bytes(290639420, 2815119, "fp32c", False) - 1.4352e9) < 1e6


def test_cpu_sample_of_batched_workload_is_its_first_specimens():
    work = configs.batched_cubes(nspec=32)
    sub, text = bench.cpu_workload(work, max_particles=60000)
    n = sum(m.general.n for m in sub["materials"])
    assert 0 < len(sub["materials"]) < 32
    assert n <= 60000 and n + work["materials"][len(sub["materials"])].general.n > 60000
    assert sub["materials"] == work["materials"][:len(sub["materials"])]
    assert text.startswith(f"first {len(sub['materials'])} of 32 specimens")
    bar = configs.lps_bar(nx=20, ny=5, nz=5)
    assert bench.cpu_workload(bar)[0] is bar


def test_compute_roofline_fractions(monkeypatch):
    """The compute object: walked slots x (29 FP32-pipe, 3 MUFU) lane
    operations over the step time, against the measured pipe rates (here a
    fake of pd_pipe_peaks: no GPU call)."""
    from peridyn_b200 import _abi

    fake = dict(zip(_abi.PIPE_KEYS, (3.5e13, 3.7e13, 4.6e12, 4.5e12, 1.1e12)))
    monkeypatch.setattr(_abi, "pipe_peaks", lambda device=0: fake)
    c = bench.compute_roofline(320_000_000, 0.5, 0)
    t = 0.5e-3
    assert c["fp32_achieved"] == 29 * 320_000_000 / t
    assert c["fp32_frac"] == c["fp32_achieved"] / 3.5e13
    # the slower MUFU operation sets the MUFU peak
    assert c["mufu_peak"] == 4.5e12 and c["mufu_frac"] == 3 * 320_000_000 / t / 4.5e12
    assert c["slots_per_launch"] == 320_000_000
    # no step time: only the measured rates
    assert set(bench.compute_roofline(1, 0.0, 0)) == {"pipe_peaks"}


def test_cube_edge_variant_draws_one_edge_per_specimen():
    w = configs.batched_cubes(nspec=6, cubes=True)
    for m in w["materials"]:
        n = round(m.general.n ** (1.0 / 3.0))
        assert n ** 3 == m.general.n
    assert w["workload"] == "batched_6_pmb_cubes"
    # the per-axis default keeps its draws (same specimens as before)
    assert configs.batched_cubes(nspec=6)["workload"] == "batched_6_pmb"


def test_serving_sample_reports_the_stream(monkeypatch):
    """The bench line's serving object: one warm-up stream of 4 small jobs,
    then the measured stream of args.jobs FP32C jobs at their Poisson
    arrival times, its latency percentiles and aggregate rate carried over
    (a fake server here: no GPU call)."""
    import types

    import peridyn_b200 as pb

    calls = []

    class FakeServer:
        def __init__(self, device, max_active):
            calls.append(("server", device, max_active))

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

    def fake_stream(srv, jobs, arrivals):
        calls.append(("stream", len(jobs), list(arrivals)))
        assert all(j["precision"] == "fp32c" for j in jobs)
        return [], {"jobs": len(jobs), "wall_s": 2.0, "latency_ms": {"p50": 10.0, "p99": 20.0, "max": 21.0},
                    "bond_updates": 8, "bond_updates_per_s": 4.0}

    monkeypatch.setattr(pb, "Server", FakeServer)
    monkeypatch.setattr(pb, "serve_stream", fake_stream)
    args = types.SimpleNamespace(jobs=3, max_active=5)
    out = bench.serving_sample(args, 0)
    assert calls[0] == ("server", 0, 5)
    assert calls[1][:2] == ("stream", 4) and calls[1][2] == [0.0] * 4  # warm-up, submitted at once
    assert calls[2][1] == 3 and calls[2][2] == sorted(calls[2][2]) and calls[2][2][-1] > 0.0
    assert out["jobs"] == 3 and out["latency_ms"]["p99"] == 20.0
    assert out["aggregate_bond_updates_per_s"] == 4.0 and out["workload"] == "serving_3_jobs_poisson50"
