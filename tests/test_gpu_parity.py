"""Whole-increment parity of the device solve with the reference.

The goldens were produced by the reference's own MaterialGrid code (see
tests/golden/make_golden.py).  Bars (FP64 GPU path vs the reference CPU solve):
  macroscopic stress <sigma>       <= 1e-9 relative, every iteration
  per-voxel fields                 <= 1e-7 max over voxels of |a_v - b_v| / |b_v|
                                    (fields near zero, d~ and P, are normalised
                                    by the field's RMS instead)
  iteration count                  equal
Mixed precision is checked against the FP64 GPU path: <sigma> <= 1e-5 relative.
L0 is an average of the inverses of the per-voxel compliance matrices
sum_s m_s (x) m_s gdot0 |r_s|^(n-1)/tau_s; with n = 20 some of them are
ill-conditioned (cond ~ 1e8), so rounding differences between any two
correct implementations are amplified there: its bar is 1e-7 relative.
"""
import numpy as np
import pytest

from vpfft_b200 import capi, MaterialGrid

pytestmark = pytest.mark.gpu

SMALL = ["c1_16", "hard_16", "odd_15x12x10", "n20_16"]


def material_of(g):
    return capi.material(gamma_dot_base=float(g["gamma_dot_base"]),
                         rate_sensitivity=int(g["rate_sensitivity"]), crss=float(g["crss0"]),
                         tau0=float(g["tau0"]), tau1=float(g["tau1"]), theta0=float(g["theta0"]),
                         theta1=float(g["theta1"]), hardening=float(g["hardening"]))


def grid_of(g, precision="fp64"):
    dims = tuple(int(x) for x in g["dims"])
    grid = MaterialGrid(*dims, material=material_of(g), precision=precision)
    grid.SendDataAndInitialize(g["R_in"], np.zeros((grid.N, 5)))
    grid.SetVoxelLength(*[float(x) for x in g["h"]])
    return grid


def voxel_rel(a, b):
    a, b = np.asarray(a).reshape(len(a), -1), np.asarray(b).reshape(len(b), -1)
    return (np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max()


def rms_rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.sqrt(np.mean(np.asarray(b) ** 2))


def run_increments(g, precision="fp64"):
    grid = grid_of(g, precision)
    e = g["edot"]
    out = []
    for s in range(int(g["nsteps"])):
        grid.InitializeComputation(e)
        L0 = grid.BuildLinearRefMediumStiffness()
        hist = grid.FixedPoint(e, int(g["max_iter"]), float(g["eps"]))
        grid.PostIncrement(e, float(g["dt"]))
        out.append((L0, hist))
    return grid, out


@pytest.mark.parametrize("name", SMALL)
def test_increments_match_reference(name, golden, lib):
    g = golden(name)
    grid, out = run_increments(g)
    off = 0
    for s, (L0, hist) in enumerate(out):
        assert len(hist) == int(g["iters"][s]), (s, len(hist), g["iters"][s])
        assert np.abs(L0 - g["L0"][s]).max() <= 1e-7 * np.abs(g["L0"][s]).max()
        ref = g["history"][off: off + len(hist)]
        off += int(g["hist_counts"][s])
        rel = np.linalg.norm(hist[:, :5] - ref[:, :5], axis=1) / np.linalg.norm(ref[:, :5], axis=1)
        assert rel.max() <= 1e-9, (s, rel.max())
        np.testing.assert_allclose(hist[:, 10:], ref[:, 10:], rtol=1e-6)  # delta_sigma, delta_eps
        assert np.abs(hist[-1, :5] - g["avg_stress"][s]).max() <= 1e-9 * np.abs(g["avg_stress"][s]).max()
    assert voxel_rel(grid.Stress(), g["sigma"]) <= 1e-7
    assert voxel_rel(grid.LagrangeMultiplier(), g["lambda"]) <= 1e-7
    assert voxel_rel(grid.Orientation(), g["R"]) <= 1e-7
    assert voxel_rel(grid.CRSS(), g["crss"]) <= 1e-7
    assert voxel_rel(grid.AccumulatedShear()[:, None], g["accshear"][:, None]) <= 1e-7
    assert rms_rel(grid.PolarizationField(), g["P_last"]) <= 1e-7
    assert rms_rel(grid.DisplacementVariation(), g["dtilde_last"]) <= 1e-7
    np.testing.assert_allclose(grid.VoxelLength(), g["voxlen"], rtol=1e-15)
    grid.close()


def test_first_iteration_fields(golden, lib):
    """Minimum slice: initialisation, L0 and ONE fixed-point iteration reproduce
    the reference's sigma, lambda, P and d~ voxel by voxel."""
    g = golden("c1_16")
    grid = grid_of(g)
    e = g["edot"]
    grid.InitializeComputation(e)
    assert voxel_rel(grid.Stress(), g["it0_sigma"]) <= 1e-10
    grid.BuildLinearRefMediumStiffness()
    grid.FixedPoint(e, 1, float(g["eps"]))
    assert rms_rel(grid.DisplacementVariation(), g["it1_dtilde"]) <= 1e-10
    assert voxel_rel(grid.Stress(), g["it1_sigma"]) <= 1e-10
    assert voxel_rel(grid.LagrangeMultiplier(), g["it1_lambda"]) <= 1e-10
    assert rms_rel(grid.PolarizationField(), g["it1_P"]) <= 1e-10
    grid.close()


def test_run_single_strain_step_api(golden, lib, tmp_path):
    """The reference-named entry points give the same answer as the phases."""
    g = golden("c1_16")
    grid = grid_of(g)
    avg = grid.RunSingleStrainStep(g["edot"], int(g["max_iter"]), float(g["dt"]), float(g["eps"]))
    assert np.abs(avg - g["avg_stress"][0]).max() <= 1e-9 * np.abs(g["avg_stress"][0]).max()
    st = grid.last_stats
    assert st.iterations == int(g["iters"][0])
    assert st.nr_not_converged >= 0
    grid.close()
    g3 = golden("hard_16")
    grid = grid_of(g3)
    rows = grid.RunVPFFT(g3["edot"], int(g3["max_iter"]), int(g3["nsteps"]), float(g3["dt"]),
                         float(g3["eps"]), str(tmp_path / "Stress_Strain.txt"))
    assert len(rows) == int(g3["nsteps"])
    for s, (_, strain, stress) in enumerate(rows):
        np.testing.assert_allclose(stress, g3["avg_stress"][s], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(strain, g3["edot"] * g3["dt"] * (s + 1), rtol=1e-14)
    assert len(open(tmp_path / "Stress_Strain.txt").read().strip().splitlines()) == 3
    grid.close()


def test_mixed_precision_error_vs_fp64(golden, lib):
    """Mixed precision (FP32 fields/FFT/Green, FP64 NR and reductions) against
    the all-FP64 GPU path on the n=20 plane-strain material: <sigma> <= 1e-5."""
    g = golden("n20_16")
    _, o64 = run_increments(g, "fp64")
    _, o32 = run_increments(g, "mixed")
    s64, s32 = o64[0][1][-1, :5], o32[0][1][-1, :5]
    assert np.linalg.norm(s32 - s64) / np.linalg.norm(s64) <= 1e-5


def test_deterministic(golden, lib):
    g = golden("odd_15x12x10")
    a, _ = run_increments(g)
    b, _ = run_increments(g)
    assert np.array_equal(a.Stress(), b.Stress())
    assert np.array_equal(a.LagrangeMultiplier(), b.LagrangeMultiplier())


def test_errors_are_returned(lib):
    from vpfft_b200 import VpfftError, fixtures

    with pytest.raises(VpfftError) as ei:
        MaterialGrid(7, 8, 8)  # 7 is not a product of 2, 3 and 5
    assert ei.value.status == capi.ERR_UNSUPPORTED_SIZE
    grid = MaterialGrid(8, 8, 8, material=capi.material(1.0, 10, 1.0))
    with pytest.raises(VpfftError) as ei:
        grid.RunSingleStrainStep(np.zeros(5), 10, 0.01, 1e-5)
    assert ei.value.status == capi.ERR_NOT_INITIALIZED
    grid.SendDataAndInitialize(fixtures.polycrystal(8, 8, 8, 3, 1))
    # zero strain rate: the reference's Sachs guess is 0/0 (Solvers.cpp:241) and
    # its fields turn NaN; here the solve stops with an error instead
    with pytest.raises(VpfftError) as ei:
        grid.RunSingleStrainStep(np.zeros(5), 10, 0.01, 1e-5)
    assert ei.value.status == capi.ERR_NONFINITE
    with pytest.raises(VpfftError):
        grid.SetVoxelLength(0.0, 1.0, 1.0)
    # the grid stays usable after an error
    avg = grid.RunSingleStrainStep(np.array([-1.06, -0.61, 0, 0, 0]), 3, 0.01, 1e-5)
    assert np.all(np.isfinite(avg))
    assert grid.last_stats.iterations == 3
    grid.close()


def test_c2_twenty_increments_with_hardening_and_texture(golden, lib):
    """The 64^3 multi-increment case (125 grains, 20 increments of uniaxial
    tension, Voce hardening and texture update), FP64, against the reference
    run field by field: every increment's <sigma> history (1e-9), L0 (1e-7),
    the mean and RMS of sigma, lambda, R and CRSS (1e-9 relative), and sampled
    voxels after increments 1, 5, 10, 15 and 20 (1e-7 max-relative)."""
    import hashlib

    from vpfft_b200 import fixtures

    g = golden("c2_64")
    dims = tuple(int(x) for x in g["dims"])
    R = fixtures.polycrystal(*dims, int(g["grains"]), int(g["seed"]))
    assert hashlib.sha256(np.ascontiguousarray(R).tobytes()).hexdigest() == str(g["R_in_sha256"])
    grid = MaterialGrid(*dims, material=material_of(g), precision="fp64")
    grid.SendDataAndInitialize(R, np.zeros((grid.N, 5)))
    e = g["edot"]
    idx = g["sample_index"]
    off = 0
    getters = {"sigma": grid.Stress, "lambda": grid.LagrangeMultiplier, "R": grid.Orientation,
               "crss": grid.CRSS}
    for s in range(int(g["nsteps"])):
        grid.InitializeComputation(e)
        L0 = grid.BuildLinearRefMediumStiffness()
        hist = grid.FixedPoint(e, int(g["max_iter"]), float(g["eps"]))
        grid.PostIncrement(e, float(g["dt"]))
        assert len(hist) == int(g["iters"][s])
        assert np.abs(L0 - g["L0"][s]).max() <= 1e-7 * np.abs(g["L0"][s]).max()
        ref = g["history"][off: off + len(hist)]
        off += int(g["hist_counts"][s])
        rel = np.linalg.norm(hist[:, :5] - ref[:, :5], axis=1) / np.linalg.norm(ref[:, :5], axis=1)
        assert rel.max() <= 1e-9, (s, rel.max())
        np.testing.assert_allclose(hist[:, 10:], ref[:, 10:], rtol=1e-6)
        for f, get in getters.items():
            full = get().reshape(grid.N, -1)
            np.testing.assert_allclose(full.mean(axis=0), g[f"inc{s}_{f}_mean"], rtol=1e-9,
                                       atol=1e-12 * np.abs(g[f"inc{s}_{f}_rms"]).max())
            np.testing.assert_allclose(np.sqrt((full ** 2).mean(axis=0)), g[f"inc{s}_{f}_rms"],
                                       rtol=1e-9)
            if f"inc{s}_{f}" in g:
                assert voxel_rel(full[idx], g[f"inc{s}_{f}"]) <= 1e-7, (s, f)
    np.testing.assert_allclose(grid.VoxelLength(), g["voxlen"], rtol=1e-14)
    grid.close()


def test_print_dumps_of_a_solved_grid(golden, lib, tmp_path):
    """MaterialGrid::Print* of the device fields: the reference's layout (z
    outermost for stress, x outermost for the Lagrange multiplier) and the
    values of the grid at 6 significant digits."""
    g = golden("c1_16")
    grid = grid_of(g)
    grid.RunSingleStrainStep(g["edot"], 3, float(g["dt"]), float(g["eps"]))
    nx, ny, nz = (int(x) for x in g["dims"])
    for name, get, zouter in (("PrintStress", grid.Stress, True),
                              ("PrintLagrangeMultiplier", grid.LagrangeMultiplier, False),
                              ("PrintPolarization", grid.PolarizationField, True),
                              ("PrintStrain", grid.DisplacementVariation, True)):
        path = tmp_path / f"{name}.txt"
        getattr(grid, name)(str(path))
        rows = [line.split() for line in path.read_text().splitlines()]
        assert len(rows) == grid.N
        ijk = np.array([[int(t) for t in r[:3]] for r in rows])
        vals = np.array([[float(t) for t in r[3:]] for r in rows])
        if vals.shape[1] == 10:  # re/im pairs; the imaginary parts are written as 0
            assert np.all(vals[:, 1::2] == 0)
            vals = vals[:, 0::2]
        expect_first = (1, 0, 0) if zouter else (0, 0, 1)
        assert tuple(ijk[1]) == expect_first
        idx = (ijk[:, 0] * ny + ijk[:, 1]) * nz + ijk[:, 2]
        ref = get()[idx]
        np.testing.assert_allclose(vals, ref, rtol=6e-6, atol=1e-300)
    grid.close()


def test_config_driven_run(lib, tmp_path):
    """vpfft_b200.run_config: the configuration file wired to MaterialGrid
    gives the same increments as the same set-up made by hand."""
    from vpfft_b200 import fixtures, run_config

    cfg = tmp_path / "run.config"
    cfg.write_text("GridDimension 8 8 4\nInputStrainRate\n  -0.5 0 0\n  0 -0.5 0\n  0 0 1\n"
                   "MaxNRIter 100\nNRTolerence 1e-5\n"
                   "TimeStep 0.01\nNumTimeIter 2\nTwoGrainInit\nCRSS 1\nGammaDotBase 1\n"
                   "RateSensitivity 10\nTau0 1\nTau1 0.5\nTheta0 20\nTheta1 1\n"
                   "HardeningMatrix 1\nMaxIter 12\nPrecision FP64\n")
    grid, rows = run_config.run(str(cfg), str(tmp_path / "out"), print_fields=True)
    assert len(rows) == 2
    lines = (tmp_path / "out" / "Stress_Strain.txt").read_text().splitlines()
    assert len(lines) == 2
    for name in ("Strain", "Stress", "LagrangeMultiplier", "Polarization"):
        assert len((tmp_path / "out" / f"{name}.txt").read_text().splitlines()) == 256
    ref = MaterialGrid(8, 8, 4, material=capi.material(1.0, 10, 1.0, 1.0, 0.5, 20.0, 1.0, 1.0),
                       precision="fp64")
    ref.SendDataAndInitialize(fixtures.two_grain(8, 8, 4))
    e = fixtures.edot_from_matrix(np.diag([-0.5, -0.5, 1.0]))
    for (_, _, s_cfg) in rows:
        s_ref = ref.RunSingleStrainStep(e, 12, 0.01, 1e-5)
        np.testing.assert_array_equal(s_cfg, s_ref)
    grid.close()
    ref.close()
