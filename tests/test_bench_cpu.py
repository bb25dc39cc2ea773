"""bench.py's CPU comparison of the batched and serving arms (no GPU): the
reference's per-edge increment costs measured on tiny RVEs, and the solves
and the trace modelled from them."""
import numpy as np

from vpfft_b200 import serving


def test_increment_costs_and_rve_baselines(lib, port):
    import bench

    costs, kind, binary = bench.cpu_increment_costs([6, 8], k_iters=2)
    assert kind in ("reference", "port")
    for e in (6, 8):
        fixed, it = costs[e]
        assert fixed >= 0.0 and it > 0.0
    trace = serving.poisson_trace(40, 500.0, 4, seed=7)
    models = {
        "batched": {"edges": [6, 8, 6, 8, 8], "iters": [100, 100, 37, 100, 2]},
        "serving": {"trace": trace, "edges": [6, 8, 8, 6], "iters": [100] * len(trace)},
    }
    out = bench.cpu_rve_baselines(models)
    cores = bench.host_cores()
    b, s = out["batched"], out["serving"]
    assert b["cores"] == cores and s["cores"] == cores
    assert np.isfinite(b["value"]) and b["value"] > 0
    assert np.isfinite(s["value"]) and s["value"] > 0
    assert 0 < s["latency_p50_s"] <= s["latency_p99_s"]
    assert set(b["per_edge"]) == {"6", "8"}
