"""Parity over ten seeded microstructures: the FP64 device solve against the
oracle (the C restatement, which tests/test_oracle.py pins bit for bit to the
reference build) run on the same inputs here, one increment each.

Workload of the CPU-runnable configuration at 12^3 so that ten oracle solves
finish in seconds: 8 periodic-Voronoi grains from seeded points, uniform random
orientations, FCC 12 {111}<110>, n = 10, gdot0 = 1, uniform CRSS 1, uniaxial
tension diag(1, -0.5, -0.5), dt = 0.005, eps = 1e-5, at most 100 iterations;
Voce hardening and the texture update run after the loop.  Bars as in
test_gpu_parity.py: iteration counts equal, <sigma> within 1e-9 relative at
every iteration, L0 within 1e-7, per-voxel stress, Lagrange multiplier,
orientation and CRSS within 1e-7."""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from oracle import refio
from vpfft_b200 import MaterialGrid, capi, fixtures

pytestmark = pytest.mark.gpu

DIMS = (12, 12, 12)
SEEDS = list(range(1, 11))


def _case(seed):
    R = fixtures.polycrystal(*DIMS, 8, seed)
    n = int(np.prod(DIMS))
    edot = fixtures.edot_from_matrix(np.diag([1.0, -0.5, -0.5]))
    return refio.Case(DIMS, R, np.zeros((n, 5)), np.ones(12),
                      refio.Material.uniform(1.0, 10, 1.0, 0.5, 20.0, 1.0), edot, nsteps=1,
                      max_iter=100, dt=0.005, eps=1e-5)


def _rel(a, b):
    a, b = np.asarray(a).reshape(len(a), -1), np.asarray(b).reshape(len(b), -1)
    return (np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max()


def test_ten_seeds_match_the_oracle(lib, port, tmp_path):
    cases = {s: _case(s) for s in SEEDS}
    with cf.ThreadPoolExecutor(max_workers=min(len(SEEDS), os.cpu_count() or 1)) as ex:
        futs = {s: ex.submit(refio.run, refio.PORT_BIN, c, str(tmp_path / str(s)))
                for s, c in cases.items()}
        outs = {s: f.result() for s, f in futs.items()}
    mat = capi.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0, tau0=1.0, tau1=0.5,
                        theta0=20.0, theta1=1.0)
    for s in SEEDS:
        c, out = cases[s], outs[s]
        hist_ref = refio.iteration_history(out, DIMS, c.edot)[0]
        L0_ref = refio.l0_per_increment(out, DIMS[0])[0]
        grid = MaterialGrid(*DIMS, material=mat, precision="fp64")
        grid.SendDataAndInitialize(c.R, c.sigma)
        grid.InitializeComputation(c.edot)
        L0 = grid.BuildLinearRefMediumStiffness()
        hist = grid.FixedPoint(c.edot, c.max_iter, c.eps)
        grid.PostIncrement(c.edot, c.dt)
        assert len(hist) == int(out["iters"][0]) == len(hist_ref), (s, len(hist), out["iters"])
        assert np.abs(L0 - L0_ref).max() <= 1e-7 * np.abs(L0_ref).max(), s
        ref = np.array([h[0] for h in hist_ref])
        rel = np.linalg.norm(hist[:, :5] - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert rel.max() <= 1e-9, (s, rel.max())
        assert _rel(grid.Stress(), out["sigma"]) <= 1e-7, s
        assert _rel(grid.LagrangeMultiplier(), out["lambda"]) <= 1e-7, s
        assert _rel(grid.Orientation(), out["R"]) <= 1e-7, s
        assert _rel(grid.CRSS(), out["crss"]) <= 1e-7, s
        grid.close()
