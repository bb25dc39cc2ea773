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


def test_reference_arm_prints_its_json_line(port):
    """bench.py --impl reference: the reference's CPU solve on the host cores,
    one JSON line with the bench keys, impl "reference", its cpu_baseline and
    an e2e without host-device copies."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True,
                       timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
