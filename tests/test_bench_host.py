"""Host logic of bench.py: the algorithmic byte model behind the roofline
(the per-bond and per-particle figures of the survey's measurement table)
and the bounded CPU sample of the batched workload."""
import bench
from peridyn_b200 import configs


def test_step_bytes_model():
    # bond-based FP32C: 4.125 B per intact directed bond, 84 B per particle
    assert bench.step_bytes(1000, 10, "fp32c", False) == 4.125 * 1000 + 84 * 10
    # FP64: 168 B per particle
    assert bench.step_bytes(1000, 10, "fp64", False) == 4.125 * 1000 + 168 * 10
    # state-based: two bond sweeps and the dilatation (8 B) per particle
    assert bench.step_bytes(1000, 10, "fp32c", True) == 2 * 4.125 * 1000 + 92 * 10
    # the C4 figure quoted in the design notes: 290,639,420 bonds, 2,815,119 particles
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
