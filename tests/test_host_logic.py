"""Host-side logic that needs no GPU: the serving stream generator, the
latency percentiles and the library's symbol table."""
import math

import numpy as np

from peridyn_b200 import configs, serving


def test_percentile_matches_numpy_linear():
    rng = np.random.default_rng(3)
    a = rng.exponential(10.0, size=137)
    for q in (0, 1, 50, 90, 99, 100):
        assert math.isclose(serving.percentile(a, q), float(np.percentile(a, q)), rel_tol=1e-12)


def test_serving_stream_is_seeded_and_bounded():
    j1, a1 = configs.serving_jobs(40, n_lo=5e3, n_hi=5e5)
    j2, a2 = configs.serving_jobs(40, n_lo=5e3, n_hi=5e5)
    assert a1 == a2 and [w["workload"] for w in j1] == [w["workload"] for w in j2]
    assert all(b > a for a, b in zip(a1, a1[1:]))
    n = np.array([w["materials"][0].general.n for w in j1])
    # cube edges round the log-uniform count; allow the rounding
    assert n.min() >= 0.7 * 5e3 and n.max() <= 1.3 * 5e5
    steps = np.array([w["nsteps"] for w in j1])
    assert steps.min() >= 500 and steps.max() <= 5000
    kinds = {w["materials"][0].specific.kind for w in j1}
    assert kinds == {0, 1}  # both PMB and state-based jobs
    # mean inter-arrival near 1/50 s
    gaps = np.diff([0.0] + a1)
    assert 0.01 < gaps.mean() < 0.04


def test_write_ovito_layout(tmp_path):
    from peridyn_b200 import io

    y = np.array([[0.0, 1.5e-5], [2.0, -3.25], [1e-3, 4.0]])
    p = tmp_path / "s.data"
    io.write_ovito(str(p), id=np.array([1, 2]), position=y, damage=np.array([0.0, 0.5]))
    lines = p.read_text().splitlines()
    assert lines[0] == "2 "
    assert lines[1] == "# damage | id | position"
    assert lines[2] == "0.0 1 0.0 2.0 0.001 "
    assert lines[3] == "0.5 2 1.5e-5 -3.25 4.0 "
