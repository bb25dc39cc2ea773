"""Grid checkpoints (vpfft_grid_snapshot / vpfft_grid_restore): a grid restored
from a snapshot continues bit for bit as the original does -- between
increments (per-voxel CRSS, texture, accumulated shear and voxel lengths from
the first increment's hardening and texture update) and in the middle of an
increment's fixed-point loop (L0, polarization and Lagrange multiplier) --
in both precisions; snapshots of other grids are refused."""
import numpy as np
import pytest

from vpfft_b200 import MaterialGrid, capi, fixtures

pytestmark = pytest.mark.gpu

DIMS = (12, 10, 8)
E1 = fixtures.edot_from_matrix(np.diag([1.0, -0.5, -0.5]))
# traceless velocity gradient with shear
E2 = fixtures.edot_from_matrix(np.array([[0.2, 0.5, 0.0], [0.1, -0.6, 0.3], [0.0, 0.2, 0.4]]))


def _material():
    return capi.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0, tau0=1.0, tau1=0.5,
                         theta0=20.0, theta1=1.0)


def _fields(g):
    return [g.Stress(), g.LagrangeMultiplier(), g.Orientation(), g.CRSS(), g.AccumulatedShear(),
            g.VoxelLength()]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restored_grid_continues_bit_for_bit(lib, precision):
    a = MaterialGrid(*DIMS, material=_material(), precision=precision)
    a.SendDataAndInitialize(fixtures.polycrystal(*DIMS, 6, 3))
    a.RunSingleStrainStep(E1, 100, 0.005, 1e-5)
    snap = a.snapshot()
    avg_a = a.RunSingleStrainStep(E2, 100, 0.005, 1e-5)

    b = MaterialGrid(*DIMS, material=_material(), precision=precision)
    b.restore(snap)
    assert b.snapshot() == snap
    avg_b = b.RunSingleStrainStep(E2, 100, 0.005, 1e-5)
    assert np.array_equal(avg_a, avg_b)
    for fa, fb in zip(_fields(a), _fields(b)):
        assert np.array_equal(fa, fb)
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restore_in_the_middle_of_the_fixed_point_loop(lib, precision):
    a = MaterialGrid(*DIMS, material=_material(), precision=precision)
    a.SendDataAndInitialize(fixtures.polycrystal(*DIMS, 6, 4))
    a.InitializeComputation(E2)
    a.BuildLinearRefMediumStiffness()
    a.FixedPoint(E2, 5, 0.0)
    snap = a.snapshot()
    hist_a = a.FixedPoint(E2, 10, 0.0)

    b = MaterialGrid(*DIMS, material=_material(), precision=precision)
    b.restore(snap)
    hist_b = b.FixedPoint(E2, 10, 0.0)
    assert np.array_equal(hist_a, hist_b)
    assert np.array_equal(a.Stress(), b.Stress())
    assert np.array_equal(a.PolarizationField(), b.PolarizationField())
    a.close()
    b.close()


def test_snapshots_of_other_grids_are_refused(lib):
    a = MaterialGrid(*DIMS, material=_material(), precision="fp64")
    a.SendDataAndInitialize(fixtures.polycrystal(*DIMS, 6, 5))
    snap = a.snapshot()
    other = MaterialGrid(8, 10, 12, material=_material(), precision="fp64")
    mixed = MaterialGrid(*DIMS, material=_material(), precision="mixed")
    for g, data in ((other, snap), (mixed, snap), (a, snap[:-8]), (a, b"not a snapshot" * 8)):
        with pytest.raises(capi.VpfftError) as ei:
            g.restore(data)
        assert ei.value.status == capi.ERR_INVALID_ARGUMENT
    for g in (a, other, mixed):
        g.close()
