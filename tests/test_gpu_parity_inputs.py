"""Parity with the reference on the input classes of the batched and serving
workloads and on the solver's less common paths (goldens made by the
reference's own code, tests/golden/make_golden.py):

  shear_16   random traceless velocity gradients (all five strain-rate
             components, shear included), a different one per increment on a
             persistent RVE, Voce hardening + texture between the increments
  shear_24   the same recipe on an edge served by the runtime-plan FFT engine
  rich_n7    n = 7 (no compile-time kernel: the runtime-exponent path),
             per-voxel random orientations and CRSS, gdot0 = 1.3, a full
             5-component strain rate, voxel lengths (1, 0.7, 1.2), 2 increments
  n1_16      the linear branch n = 1 (Solvers.cpp:66, 177-180)

Each runs FP64 through the single-grid phases and, separately, through the
batch engine (vpfft_batch_*), and is compared with the reference run.  Bars as
in test_gpu_parity.py: iteration counts equal, <sigma> within 1e-9 relative at
every iteration (single grid) and at the end of each increment (batch), L0
within 1e-7, per-voxel fields within 1e-7 max-relative."""
import numpy as np
import pytest

import vpfft_b200 as vp
from vpfft_b200 import MaterialGrid, capi, fixtures

pytestmark = pytest.mark.gpu

CASES = ["shear_16", "shear_24", "rich_n7", "n1_16"]


def material_of(g):
    return capi.material(gamma_dot_base=float(g["gamma_dot_base"]),
                         rate_sensitivity=int(g["rate_sensitivity"]), crss=float(g["crss0"]),
                         tau0=float(g["tau0"]), tau1=float(g["tau1"]), theta0=float(g["theta0"]),
                         theta1=float(g["theta1"]), hardening=float(g["hardening"]))


def edot_of(g, s):
    return g["edot_steps"][s] if "edot_steps" in g else g["edot"]


def setup(grid, g):
    grid.SendDataAndInitialize(g["R_in"], np.zeros((grid.N, 5)))
    if "crss_in" in g:
        grid.SetCRSS(g["crss_in"])
    grid.SetVoxelLength(*[float(x) for x in g["h"]])
    return grid


def voxel_rel(a, b):
    a, b = np.asarray(a).reshape(len(a), -1), np.asarray(b).reshape(len(b), -1)
    return (np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max()


def check_fields(grid, g):
    assert voxel_rel(grid.Stress(), g["sigma"]) <= 1e-7
    assert voxel_rel(grid.LagrangeMultiplier(), g["lambda"]) <= 1e-7
    assert voxel_rel(grid.Orientation(), g["R"]) <= 1e-7
    assert voxel_rel(grid.CRSS(), g["crss"]) <= 1e-7
    assert voxel_rel(grid.AccumulatedShear()[:, None], g["accshear"][:, None]) <= 1e-7
    np.testing.assert_allclose(grid.VoxelLength(), g["voxlen"], rtol=1e-14)


@pytest.mark.parametrize("name", CASES)
def test_single_grid_matches_reference(name, golden, lib):
    g = golden(name)
    dims = tuple(int(x) for x in g["dims"])
    grid = setup(MaterialGrid(*dims, material=material_of(g), precision="fp64"), g)
    off = 0
    for s in range(int(g["nsteps"])):
        e = edot_of(g, s)
        grid.InitializeComputation(e)
        if s == 0 and "it0_sigma" in g:
            assert voxel_rel(grid.Stress(), g["it0_sigma"]) <= 1e-10
        L0 = grid.BuildLinearRefMediumStiffness()
        hist = grid.FixedPoint(e, int(g["max_iter"]), float(g["eps"]))
        grid.PostIncrement(e, float(g["dt"]))
        assert len(hist) == int(g["iters"][s]), (s, len(hist), g["iters"][s])
        assert np.abs(L0 - g["L0"][s]).max() <= 1e-7 * np.abs(g["L0"][s]).max()
        ref = g["history"][off: off + len(hist)]
        off += int(g["hist_counts"][s])
        rel = np.linalg.norm(hist[:, :5] - ref[:, :5], axis=1) / np.linalg.norm(ref[:, :5], axis=1)
        assert rel.max() <= 1e-9, (s, rel.max())
        np.testing.assert_allclose(hist[:, 5:10], ref[:, 5:10], rtol=1e-9,
                                   atol=1e-9 * np.abs(ref[:, 5:10]).max())
        # delta_sigma and delta_eps are relative norms: at rounding level (the
        # linear n = 1 case, where sigma = lambda to the last bits) compare absolutely
        np.testing.assert_allclose(hist[:, 10:], ref[:, 10:], rtol=1e-6, atol=1e-12)
    check_fields(grid, g)
    grid.close()


@pytest.mark.parametrize("name", CASES)
def test_batched_fp64_matches_reference(name, golden, lib):
    """The same increments as requests to the batch engine, beside two other
    RVEs of different sizes in flight (so the batched kernels decode several
    slots), against the reference."""
    g = golden(name)
    dims = tuple(int(x) for x in g["dims"])
    mat = material_of(g)
    with vp.Batch(precision="fp64", material=mat, max_slots=4, iterations_per_tick=8) as b:
        grid = setup(b.new_grid(*dims), g)
        others = []
        for k, od in enumerate([(8, 8, 8), (20, 12, 10)]):
            o = b.new_grid(*od)
            o.SendDataAndInitialize(fixtures.polycrystal(*od, 3 + k, 40 + k))
            others.append(o)
        for s in range(int(g["nsteps"])):
            rid = b.submit(grid, edot_of(g, s), int(g["max_iter"]), float(g["dt"]),
                           float(g["eps"]))
            for o in others:
                b.submit(o, edot_of(g, s), 20, 0.005, 1e-5)
            b.run()
            res = {r.request_id: r for r in b.poll()}[rid]
            assert res.status == capi.OK
            assert res.iterations == int(g["iters"][s]), (s, res.iterations, g["iters"][s])
            ref = g["avg_stress"][s]
            assert np.linalg.norm(res.avg_stress - ref) <= 1e-9 * np.linalg.norm(ref), s
        check_fields(grid, g)
        for o in others:
            o.close()
        grid.close()


def test_stress_strain_file_matches_reference(lib, tmp_path):
    """Stress_Strain.txt from vpfft_run (RunVPFFT) is byte-identical to the one
    the reference's RunVPFFT wrote for the same inputs (MaterialGrid.cpp:
    1217-1226: step, strain, <sigma>, the two norms, 6 significant digits)."""
    import os

    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import STRESS_STRAIN as c, case_inputs

    ref_path = os.path.join(os.path.dirname(__file__), "golden", "io", "stress_strain_16.txt")
    R, crss, _, edot, _, _ = case_inputs(c)
    mat = capi.material(gamma_dot_base=1.0, rate_sensitivity=c["n"], crss=1.0, tau0=1.0,
                        tau1=0.5, theta0=20.0, theta1=1.0, hardening=1.0)
    grid = MaterialGrid(*c["dims"], material=mat, precision="fp64")
    grid.SendDataAndInitialize(R, np.zeros((grid.N, 5)))
    out = tmp_path / "Stress_Strain.txt"
    grid.RunVPFFT(edot, c["max_iter"], c["nsteps"], c["dt"], c["eps"], str(out))
    grid.close()
    assert out.read_bytes() == open(ref_path, "rb").read()
