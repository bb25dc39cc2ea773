"""Host logic of the serving loop (no GPU): the synthetic arrival trace."""
import numpy as np

from vpfft_b200 import fixtures, serving


def test_poisson_trace_statistics(lib):
    tr = serving.poisson_trace(4000, 500.0, 64, seed=3)
    t = np.array([r.t_arrival for r in tr])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 500.0) < 0.05 / 500.0          # mean inter-arrival 2 ms
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.06           # exponential: CV = 1
    counts = np.bincount([r.rve for r in tr], minlength=64)
    assert counts.min() > 0 and counts.max() < 3 * counts.mean()  # uniform over the pool
    for r in tr[:50]:
        D = 0.5 * (r.L + r.L.T)
        assert abs(np.trace(r.L)) < 1e-12
        assert abs(np.sqrt(2.0 / 3.0 * np.sum(D * D)) - 1.0) < 1e-12
        np.testing.assert_allclose(r.edot, fixtures.edot_from_matrix(r.L), rtol=0, atol=0)
    # seeded: the same trace twice
    tr2 = serving.poisson_trace(4000, 500.0, 64, seed=3)
    assert all(a.t_arrival == b.t_arrival and a.rve == b.rve for a, b in zip(tr, tr2))
