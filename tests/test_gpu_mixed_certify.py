"""The mixed-precision NR sweep's FP64 residual certificate and its FP64-step queue.

In mixed precision each voxel's FP32 Newton predictor is followed by the FP64
residual at the predicted stress; where the Newton step it asks for is below
vpfft_solver_options.mixed_certify_step x |sigma| the predicted stress is kept,
elsewhere the voxel is queued and takes the FP64 Newton step (FP64 residual
and Jacobian) with 31 other queued voxels of its warp.  With the bound at 0
every voxel-iteration takes the step through the queue, so these tests drive
both branches:

- stats.nr_fp64_steps counts the voxel-iterations that took the step: all of
  them at bound 0, few at the default;
- with either bound, <sigma> stays within 1e-5 relative of the all-FP64 path at
  every iteration (the mixed path's stated bar), and the two bounds agree with
  each other to 1e-6;
- results are the same bit for bit run to run (the queue order is fixed);
- the batched sweep, which runs the same body, gives each RVE what the
  single-grid sweep gives it at bound 0 (1e-12, the batch tests' bar);
- on per-voxel CRSS (the increment after a hardening update) the mixed path
  stays within 1e-5 of the FP64 path."""
import numpy as np
import pytest

import vpfft_b200 as vp
from vpfft_b200 import capi, fixtures

pytestmark = pytest.mark.gpu

DIMS, GRAINS, SEED, ITERS = (32, 24, 20), 12, 77, 10


def material(n=20):
    return vp.material(gamma_dot_base=1.0, rate_sensitivity=n, crss=1.0, tau0=1.0, tau1=0.5,
                       theta0=20.0, theta1=1.0)


def run(precision, certify=None, n=20, dims=DIMS):
    R = fixtures.polycrystal(*dims, GRAINS, SEED)
    e = fixtures.edot_from_matrix(np.diag([1.0, 0.0, -1.0]))
    opts = capi.solver_options(mixed_certify_step=certify) if certify is not None else None
    g = vp.MaterialGrid(*dims, material=material(n), precision=precision, options=opts)
    g.SendDataAndInitialize(R, None)
    g.InitializeComputation(e)
    g.BuildLinearRefMediumStiffness()
    hist = g.FixedPoint(e, ITERS, 0.0)
    out = (hist, g.Stress(), int(g.last_stats.nr_fp64_steps))
    g.close()
    return out


# (15, 12, 10): 1800 voxels, not a multiple of 32, so the last warp of the
# sweep is partial and its queue is flushed part-full
@pytest.mark.parametrize("n,dims", [(20, DIMS), (7, DIMS), (20, (15, 12, 10))])
def test_certified_and_queued_steps_against_fp64(lib, n, dims):
    nvox = int(np.prod(dims))
    h64, s64, k64 = run("fp64", n=n, dims=dims)
    assert k64 == 0
    hd, sd, kd = run("mixed", n=n, dims=dims)
    h0, s0, k0 = run("mixed", 0.0, n=n, dims=dims)
    assert k0 == nvox * ITERS  # bound 0: every voxel-iteration took the FP64 step
    assert 0 <= kd < k0
    print(f"\nn={n}: FP64 steps per voxel-iteration, default bound {kd / (nvox * ITERS):.2e}")
    for h in (hd, h0):
        rel = np.linalg.norm(h[:, :5] - h64[:, :5], axis=1) / np.linalg.norm(h64[:, :5], axis=1)
        assert rel.max() <= 1e-5, rel
    rel = np.linalg.norm(hd[:, :5] - h0[:, :5], axis=1) / np.linalg.norm(h0[:, :5], axis=1)
    assert rel.max() <= 1e-6, rel
    vox = np.linalg.norm(sd - s0, axis=1) / np.linalg.norm(s0, axis=1)
    assert np.percentile(vox, 99) <= 1e-4


def test_queue_deterministic(lib):
    a = run("mixed", 0.0)
    b = run("mixed", 0.0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    c = run("mixed")
    d = run("mixed")
    assert np.array_equal(c[0], d[0]) and np.array_equal(c[1], d[1]) and c[2] == d[2]


def test_batched_queue_equals_single_grid(lib):
    """Bound 0 in a batch of three RVEs (the batched sweep's queue) against the
    same RVEs alone on the single-grid path."""
    opts = capi.solver_options(mixed_certify_step=0.0)
    mat = material(10)
    dims = [(16, 16, 16), (24, 20, 18), (32, 32, 32)]

    def edot(i):
        rng = np.random.default_rng(300 + i)
        return fixtures.edot_from_matrix(fixtures.random_traceless_velocity_gradient(rng))

    def grid(d, i, factory):
        g = factory(*d)
        g.SendDataAndInitialize(fixtures.polycrystal(*d, 5 + i, 40 + i))
        return g

    with vp.Batch("mixed", material=mat, options=opts, iterations_per_tick=4) as b:
        gs = [grid(d, i, b.new_grid) for i, d in enumerate(dims)]
        ids = [b.submit(g, edot(i), 12, 0.005, 1e-5) for i, g in enumerate(gs)]
        b.run()
        res = {r.request_id: r for r in b.poll()}
        for i, d in enumerate(dims):
            alone = vp.MaterialGrid(*d, material=mat, precision="mixed", options=opts)
            alone.SendDataAndInitialize(fixtures.polycrystal(*d, 5 + i, 40 + i))
            avg = alone.RunSingleStrainStep(edot(i), 12, 0.005, 1e-5)
            r = res[ids[i]]
            assert r.iterations == alone.last_stats.iterations
            assert np.abs(r.avg_stress - avg).max() <= 1e-12 * np.abs(avg).max()
            s_b, s_a = gs[i].Stress(), alone.Stress()
            assert np.abs(s_b - s_a).max() <= 1e-12 * np.abs(s_a).max()
            alone.close()
        for g in gs:
            g.close()


def test_per_voxel_crss_increments_against_fp64(lib):
    """Two increments with Voce hardening: the second runs on per-voxel CRSS, so
    the mixed sweep stages 1/CRSS per voxel (FP32 reciprocal) beside the Schmid
    vectors; <sigma> of each increment within 1e-5 of the FP64 path."""
    R = fixtures.polycrystal(*DIMS, GRAINS, SEED)
    e = fixtures.edot_from_matrix(np.diag([1.0, -0.5, -0.5]))
    out = {}
    for prec in ("fp64", "mixed"):
        g = vp.MaterialGrid(*DIMS, material=material(10), precision=prec)
        g.SendDataAndInitialize(R, None)
        out[prec] = [g.RunSingleStrainStep(e, 30, 0.005, 0.0) for _ in range(2)]
        crss = g.CRSS()
        g.close()
        assert np.ptp(crss) > 0  # the CRSS differs between voxels after the first increment
    for a64, a32 in zip(out["fp64"], out["mixed"]):
        assert np.linalg.norm(a32 - a64) / np.linalg.norm(a64) <= 1e-5
