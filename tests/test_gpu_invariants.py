"""Invariants of the fixed-point iteration on the device fields.

- <d~> = 0: the Green operator is zero at k = 0 (MaterialGrid.cpp:733-740), so
  the strain-rate variation has zero mean.
- |<edot> - Edot| <= delta_eps |Edot| at every iteration: with <d~> = 0,
  <edot> - Edot is the mean of edot - Edot - d~ over the voxels, and the norm
  of a mean is at most the mean of the norms, which is what delta_eps
  measures (MaterialGrid.cpp:1009-1053)."""
import numpy as np
import pytest

from vpfft_b200 import MaterialGrid, capi, fixtures

pytestmark = pytest.mark.gpu

DIMS = (12, 10, 8)
# slack for rounding: FP64 fields, or FP32 fields and spectra (mixed)
TOL = {"fp64": 1e-12, "mixed": 1e-5}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zero_mean_variation_and_mean_strain_rate_bound(lib, precision):
    mat = capi.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0)
    g = MaterialGrid(*DIMS, material=mat, precision=precision)
    g.SendDataAndInitialize(fixtures.polycrystal(*DIMS, 6, 8))
    e = fixtures.edot_from_matrix(np.diag([1.0, -0.5, -0.5]))
    g.InitializeComputation(e)
    g.BuildLinearRefMediumStiffness()
    hist = g.FixedPoint(e, 6, 0.0)
    d = g.DisplacementVariation()
    rms = np.sqrt(np.mean(d ** 2))
    assert rms > 0
    assert np.abs(d.mean(axis=0)).max() <= TOL[precision] * rms
    en = np.linalg.norm(e)
    for row in hist:
        gap = np.linalg.norm(row[5:10] - e)
        assert gap <= row[11] * en * (1 + TOL[precision]) + TOL[precision] * en
    g.close()
