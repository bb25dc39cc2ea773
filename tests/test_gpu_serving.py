"""The serving loop: a Poisson stream of one-increment requests on a pool of
persistent RVEs, continuously batched.  Every request's result must equal the
same request replayed alone, in arrival order per RVE, on a twin pool through
the single-grid path (RunSingleStrainStep).  Bar: <sigma> within 1e-12
relative, equal iteration counts; the final fields of every pool RVE within
1e-12 of its twin's."""
import numpy as np
import pytest

import vpfft_b200 as vp
from vpfft_b200 import capi, serving

pytestmark = pytest.mark.gpu

TOL = 1e-12


def material():
    return vp.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0, tau0=1.0, tau1=0.5,
                       theta0=20.0, theta1=1.0)


def test_served_results_equal_requests_replayed_alone(lib):
    mat = material()
    with vp.Batch("mixed", material=mat, max_slots=3, iterations_per_tick=2) as b, \
         vp.Batch("mixed", material=mat) as twin_factory:
        pool = serving.rve_pool(b, [8, 12, 16], [0.4, 0.3, 0.3], 4, seed=5, grains=(3, 9))
        twins = serving.rve_pool(twin_factory, [8, 12, 16], [0.4, 0.3, 0.3], 4, seed=5,
                                 grains=(3, 9))
        trace = serving.poisson_trace(24, 2000.0, len(pool), seed=6)
        out = serving.serve(b, pool, trace, max_iter=60, eps=1e-4)
        assert out["completed_ok"] == len(trace)
        assert out["latency_p99_s"] >= out["latency_p50_s"] > 0
        for k, req in enumerate(trace):
            r = out["results"][k]
            assert r.status == capi.OK
            avg = twins[req.rve].RunSingleStrainStep(req.edot, 60, 0.005, 1e-4)
            assert r.iterations == twins[req.rve].last_stats.iterations, k
            assert np.abs(r.avg_stress - avg).max() <= TOL * np.abs(avg).max(), k
        for g, t in zip(pool, twins):
            for a, c in ((g.Stress(), t.Stress()), (g.Orientation(), t.Orientation()),
                         (g.CRSS(), t.CRSS())):
                assert np.abs(a - c).max() <= TOL * np.abs(c).max()
