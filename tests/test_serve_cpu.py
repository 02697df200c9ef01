"""Host-side pieces of the serving loop and the uneven workload (no GPU)."""
import numpy as np


def test_arrivals_and_percentiles():
    from neko_b200 import serve
    t = serve.arrivals(1000.0, 20000, seed=3)
    assert np.all(np.diff(t) >= 0)
    assert abs(t[-1] / 20000 - 1e-3) < 5e-5  # mean gap 1/rate
    p = serve.percentiles([0.001 * i for i in range(1, 101)])
    assert abs(p["p50_ms"] - 50.5) < 1e-9 and p["max_ms"] == 100.0
    assert p["p50_ms"] <= p["p95_ms"] <= p["p99_ms"] <= p["max_ms"]


def test_uneven_specs_distribution():
    from neko_b200 import workloads
    s = workloads.uneven_specs(4000, seed=4)
    ns = np.array([x["n"] for x in s])
    assert ns.min() == 2 and ns.max() == 16
    assert set(x["lx"] for x in s) == {6, 8, 10}
    h1 = np.array([x["h1"] for x in s])
    h2 = np.array([x["h2"] for x in s])
    assert 0.5 <= h1.min() and h1.max() <= 2.0 and 0.0 <= h2.min() and h2.max() <= 100.0
    assert len({x["dseed"] for x in s}) == workloads.N_DEFORM_SEEDS
    amps = [workloads.deform_amplitude(d) for d in range(workloads.N_DEFORM_SEEDS)]
    assert all(0.0 <= a <= 0.1 for a in amps)
    assert workloads.uneven_specs(10, seed=4) == s[:10]  # seeded, prefix-stable
