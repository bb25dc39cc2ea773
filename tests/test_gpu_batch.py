"""The batch engine (vpfft_batch_*): RVEs of different sizes advanced together
must give each RVE the same result as solving it alone with the single-grid
path (RunSingleStrainStep through vpfft_run_single_strain_step).

Bar: the batched kernels run the same per-voxel and per-wave-vector code with
the same per-RVE block partition, so results agree to rounding: <sigma> and
every field within 1e-12 relative (max over voxels of |a - b| / max|b|), equal
iteration counts.  Checked for FP64 and mixed precision, alone vs in the mix,
for a persistent RVE over two increments, with few slots (continuous
admission), under a tight HBM budget, with CUDA-graph replay, and for
cancellation and the busy-grid guard."""
import numpy as np
import pytest

import vpfft_b200 as vp
from vpfft_b200 import capi, fixtures

pytestmark = pytest.mark.gpu

TOL = 1e-12
# cubic and non-cubic RVEs: compile-time line engines (16, 32, 48, 64), the
# runtime-plan engine (8, 10, 12, 18, 20, 24) and both on different axes, so
# the batch forms several size classes whose pass chains run concurrently
DIMS = [(16, 16, 16), (12, 10, 8), (24, 20, 18), (32, 32, 32), (8, 8, 8), (48, 16, 20),
        (16, 64, 32)]


def material():
    return vp.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0, tau0=1.0, tau1=0.5,
                       theta0=20.0, theta1=1.0)


def edot_for(i):
    rng = np.random.default_rng(100 + i)
    return fixtures.edot_from_matrix(fixtures.random_traceless_velocity_gradient(rng))


def make_grid(dims, i, precision, factory=None):
    R = fixtures.polycrystal(*dims, 4 + 3 * i, 7 + i)
    g = factory(*dims) if factory else vp.MaterialGrid(*dims, material=material(),
                                                       precision=precision)
    g.SendDataAndInitialize(R)
    return g


def fields(g):
    return {"stress": g.Stress(), "lambda": g.LagrangeMultiplier(), "R": g.Orientation(),
            "crss": g.CRSS(), "acc": g.AccumulatedShear()}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def assert_same(res_avg, res_iters, g_batch, ref_avg, ref_iters, g_ref, what):
    assert res_iters == ref_iters, (what, res_iters, ref_iters)
    assert rel(res_avg, ref_avg) <= TOL, (what, rel(res_avg, ref_avg))
    fb, fr = fields(g_batch), fields(g_ref)
    for k in fr:
        assert rel(fb[k], fr[k]) <= TOL, (what, k, rel(fb[k], fr[k]))


def solve_alone(dims, i, precision, steps=1):
    g = make_grid(dims, i, precision)
    avgs, iters = [], []
    for _ in range(steps):
        avgs.append(g.RunSingleStrainStep(edot_for(i), 100, 0.005, 1e-5))
        iters.append(g.last_stats.iterations)
    return g, avgs, iters


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_grid_for_every_rve(lib, precision):
    with vp.Batch(precision, material=material(), iterations_per_tick=4) as b:
        grids, ids = [], []
        for i, d in enumerate(DIMS):
            g = make_grid(d, i, precision, b.new_grid)
            grids.append(g)
            ids.append(b.submit(g, edot_for(i), 100, 0.005, 1e-5))
        b.run()
        res = {r.request_id: r for r in b.poll()}
        assert sorted(res) == sorted(ids)
        info = b.info()
        assert info["graph_replays"] > 0  # the iteration chunk was replayed from a graph
        for i, d in enumerate(DIMS):
            r = res[ids[i]]
            assert r.status == capi.OK
            ref, avgs, iters = solve_alone(d, i, precision)
            assert r.converged == bool(ref.last_stats.converged)
            assert_same(r.avg_stress, r.iterations, grids[i], avgs[0], iters[0], ref,
                        f"{precision} rve {i} {d}")


def test_result_same_alone_and_in_the_mix(lib):
    """One RVE solved in a batch by itself and in a batch with four others."""
    d, i = DIMS[2], 2
    with vp.Batch("mixed", material=material()) as b:
        g1 = make_grid(d, i, "mixed", b.new_grid)
        b.submit(g1, edot_for(i))
        b.run()
        (r1,) = b.poll()
        g2 = make_grid(d, i, "mixed", b.new_grid)
        others = [make_grid(dd, j, "mixed", b.new_grid) for j, dd in enumerate(DIMS) if j != i]
        for j, o in zip([j for j in range(len(DIMS)) if j != i], others):
            b.submit(o, edot_for(j))
        rid = b.submit(g2, edot_for(i))
        b.run()
        r2 = {r.request_id: r for r in b.poll()}[rid]
        assert_same(r2.avg_stress, r2.iterations, g2, r1.avg_stress, r1.iterations, g1, "mix")


def test_persistent_rve_two_increments_fifo(lib):
    """Two requests on the same grid run one after the other (texture and CRSS
    carry over) and match two single-grid increments."""
    d, i = DIMS[0], 0
    with vp.Batch("fp64", material=material()) as b:
        g = make_grid(d, i, "fp64", b.new_grid)
        id1 = b.submit(g, edot_for(i))
        id2 = b.submit(g, edot_for(i))
        b.run()
        res = {r.request_id: r for r in b.poll()}
        ref, avgs, iters = solve_alone(d, i, "fp64", steps=2)
        assert res[id1].iterations == iters[0]
        assert rel(res[id1].avg_stress, avgs[0]) <= TOL
        assert_same(res[id2].avg_stress, res[id2].iterations, g, avgs[1], iters[1], ref, "inc2")


def test_few_slots_and_tight_budget_admit_continuously(lib):
    """max_slots = 2 and an HBM budget that holds the spectra of one 32^3 RVE:
    requests wait for slots and memory, and every result still matches."""
    prec = "mixed"
    spec32 = 2 * 4 * 5 * 32 * 32 * 17  # one spectrum buffer of a 32^3 mixed grid
    with vp.Batch(prec, material=material(), max_slots=2, iterations_per_tick=2,
                  hbm_budget_bytes=2 * spec32 + 4096) as b:
        grids, ids = [], []
        for i, d in enumerate(DIMS):
            g = make_grid(d, i, prec, b.new_grid)
            grids.append(g)
            ids.append(b.submit(g, edot_for(i)))
        ticks = 0
        while b.step():
            ticks += 1
            assert b.info()["active"] <= 2
        info = b.info()
        assert info["admissions_deferred_for_memory"] > 0
        assert info["arena_bytes_in_use"] == 0
        res = {r.request_id: r for r in b.poll()}
        for i, d in enumerate(DIMS):
            ref, avgs, iters = solve_alone(d, i, prec)
            assert_same(res[ids[i]].avg_stress, res[ids[i]].iterations, grids[i], avgs[0],
                        iters[0], ref, f"rve {i}")


def test_cancel_and_busy_grid(lib):
    with vp.Batch("mixed", material=material(), max_slots=1) as b:
        g1 = make_grid(DIMS[0], 0, "mixed", b.new_grid)
        g2 = make_grid(DIMS[1], 1, "mixed", b.new_grid)
        id1 = b.submit(g1, edot_for(0))
        id2 = b.submit(g2, edot_for(1))
        b.step()  # g1 admitted (one slot), g2 queued
        with pytest.raises(capi.VpfftError) as e:
            g1.Stress()
        assert e.value.status == capi.ERR_BUSY
        b.cancel(id2)
        b.cancel(id1)
        b.run()
        res = {r.request_id: r for r in b.poll()}
        assert res[id1].status == capi.ERR_CANCELLED
        assert res[id2].status == capi.ERR_CANCELLED
        g1.Stress()  # usable again
        # the grid can take a new request after the cancellation
        id3 = b.submit(g2, edot_for(1))
        b.run()
        (r3,) = b.poll()
        assert r3.request_id == id3 and r3.status == capi.OK


def test_submit_rejects_mismatched_grid(lib):
    with vp.Batch("mixed", material=material()) as b:
        g = vp.MaterialGrid(8, 8, 8, material=material(), precision="fp64")
        g.SendDataAndInitialize(fixtures.polycrystal(8, 8, 8, 3, 1))
        with pytest.raises(capi.VpfftError):
            b.submit(g, edot_for(0))
        g2 = vp.MaterialGrid(8, 8, 8, material=vp.material(), precision="mixed")
        with pytest.raises(capi.VpfftError):
            b.submit(g2, edot_for(0))


# edges with several batched tile families (compile-time engines up to 96
# points), one axis with the runtime-plan engine, and a 96-point axis
TILE_DIMS = [(16, 16, 16), (32, 48, 16), (64, 32, 48), (24, 16, 32), (96, 16, 16)]
# Every tile family (and the single-grid tiles) runs the same arithmetic: the
# line transforms and the Green operator spell out their fused multiply-adds
# and their units are built without contraction, so results agree bit for bit
# in both precisions.


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fft_tile_families_and_autotuner(lib, precision):
    """Forced tile families and the autotuned choice: results are the same bit
    for bit in every family, in FP64 and in mixed precision; the tuning record
    lists each admitted size once, in admission order, with the timed chain of
    every family and the fastest one chosen."""
    runs = {}
    for tiles in (2, -1, 0, 1):
        with vp.Batch(precision, material=material(), iterations_per_tick=4,
                      fft_tiles=tiles) as b:
            grids, ids = [], []
            for i, d in enumerate(TILE_DIMS):
                g = make_grid(d, i, precision, b.new_grid)
                grids.append(g)
                ids.append(b.submit(g, edot_for(i), 100, 0.005, 1e-5))
            b.run()
            res = {r.request_id: r for r in b.poll()}
            tun = b.tunings()
            runs[tiles] = [(res[ids[i]], fields(grids[i])) for i in range(len(TILE_DIMS))]
        assert [t["dims"] for t in tun] == TILE_DIMS
        for t in tun:
            assert 0 <= t["fft_tiles"] < t["families"]
            if tiles >= 0:
                assert t["source"] == "options"
                assert t["fft_tiles"] == min(tiles, t["families"] - 1)
            else:
                assert t["source"] in ("timed", "cached")
                ms = t["ms_per_chain"]
                assert len(ms) == t["families"] and min(ms) > 0
                assert t["fft_tiles"] == int(np.argmin(ms))
        # fixed engines up to 96 points: three families in FP32, two in FP64
        fams = {t["dims"]: t["families"] for t in tun}
        assert fams[(16, 16, 16)] == (3 if precision == "mixed" else 2)
    worst = {}
    for tiles in (-1, 0, 1):
        for i, d in enumerate(TILE_DIMS):
            (ra, fa), (rb, fb) = runs[2][i], runs[tiles][i]
            assert ra.status == capi.OK and rb.status == capi.OK
            assert ra.iterations == rb.iterations, (tiles, d)
            worst[(tiles, d, "avg")] = rel(rb.avg_stress, ra.avg_stress)
            for k in fa:
                worst[(tiles, d, k)] = rel(fb[k], fa[k])
    assert max(worst.values()) == 0.0, max(worst.items(), key=lambda kv: kv[1])
