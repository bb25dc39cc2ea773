"""Host logic of the serving loop and of the CPU comparison (no GPU): the
synthetic arrival trace, the RVE pool draws, the FIFO replay and the
longest-first packing of independent solves."""
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


def test_pool_specs_seeded_and_weighted(lib):
    a = serving.pool_specs([32, 48, 64, 96], [0.4, 0.3, 0.2, 0.1], 2000, seed=5)
    assert a == serving.pool_specs([32, 48, 64, 96], [0.4, 0.3, 0.2, 0.1], 2000, seed=5)
    edges = np.array([e for e, _ in a])
    grains = np.array([g for _, g in a])
    for e, w in ((32, 0.4), (48, 0.3), (64, 0.2), (96, 0.1)):
        assert abs(np.mean(edges == e) - w) < 0.04
    assert grains.min() >= 8 and grains.max() <= 200


def test_fifo_replay_hand_case(lib):
    def req(t, rve):
        return serving.Request(t, rve, np.zeros((3, 3)))

    # two workers, unit service times; the third request waits for its RVE's
    # first increment and for a free worker
    tr = [req(0.0, 0), req(0.1, 1), req(0.2, 0), req(0.3, 2)]
    r = serving.fifo_replay(tr, [1.0, 1.0, 1.0, 1.0], 2)
    np.testing.assert_allclose(r["latency_max_s"], 1.8)
    np.testing.assert_allclose(r["latency_p50_s"], np.quantile([1.0, 1.0, 1.8, 1.8], 0.5))
    np.testing.assert_allclose(r["throughput"], 4 / 2.1)
    # the same RVE twice: the second increment starts when the first ends,
    # even with a worker free
    r = serving.fifo_replay([req(0.0, 3), req(0.0, 3)], [1.0, 1.0], 2)
    np.testing.assert_allclose(r["latency_max_s"], 2.0)


def test_lpt_makespan(lib):
    import bench

    assert bench.lpt_makespan([4.0, 3.0, 2.0, 1.0], 2) == 5.0
    assert bench.lpt_makespan([1.0] * 10, 3) == 4.0
    assert bench.lpt_makespan([2.0, 7.0], 16) == 7.0
