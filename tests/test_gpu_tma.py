"""The y and z passes with tiles moved by the Tensor Memory Accelerator
(vpfft_b200/csrc/fft_tma.cu) against the warp-copy passes: the same line
transforms on the same lines, so the results must be the same bit for bit.
Checked through the forward and inverse 3D transform entry points (FP32) on
grids whose y or z lines take the TMA path (64, 128 and 256 points) and grids
where only some passes do, and through a whole mixed-precision fixed-point run
(every iteration's <sigma> and the final fields equal bit for bit with the
switch on and off)."""
import ctypes as C

import numpy as np
import pytest

import vpfft_b200 as vp
from vpfft_b200 import capi, fixtures

pytestmark = pytest.mark.gpu


@pytest.fixture
def tma(lib):
    prev = lib.vpfft_set_tma_passes(-1)
    yield lib
    lib.vpfft_set_tma_passes(prev)


def _r2c(lib, dims, real):
    nx, ny, nz = dims
    spec = np.zeros(5 * nx * ny * (nz // 2 + 1) * 2)
    capi.check(lib.vpfft_fft3d_r2c(nx, ny, nz, 5, capi.dptr(real), capi.dptr(spec),
                                   capi.PREC_MIXED))
    return spec


DIMS = [(64, 64, 32), (32, 128, 16), (16, 256, 8), (96, 64, 48), (16, 32, 256), (8, 64, 128),
        (32, 64, 64), (12, 20, 256)]


@pytest.mark.parametrize("dims", DIMS)
def test_forward_transform_same_bits(tma, dims):
    real = np.random.default_rng(7).normal(size=5 * int(np.prod(dims)))
    tma.vpfft_set_tma_passes(0)
    ref = _r2c(tma, dims, real)
    tma.vpfft_set_tma_passes(1)
    got = _r2c(tma, dims, real)
    assert np.array_equal(got, ref)
    # and it is the transform: against numpy's at FP32 accuracy
    nx, ny, nz = dims
    want = np.fft.rfftn(real.reshape(5, nx, ny, nz), axes=(1, 2, 3))
    spec = got.reshape(5, nx, ny, nz // 2 + 1, 2)
    err = np.abs(spec[..., 0] + 1j * spec[..., 1] - want).max() / np.abs(want).max()
    assert err < 3e-6, err


def _c2r(lib, dims, spec):
    nx, ny, nz = dims
    real = np.zeros(5 * nx * ny * nz)
    capi.check(lib.vpfft_fft3d_c2r(nx, ny, nz, 5, capi.dptr(spec), capi.dptr(real),
                                   capi.PREC_MIXED))
    return real


@pytest.mark.parametrize("dims", DIMS)
def test_inverse_transform_same_bits(tma, dims):
    nx, ny, nz = dims
    real = np.random.default_rng(8).normal(size=5 * nx * ny * nz)
    tma.vpfft_set_tma_passes(0)
    spec = _r2c(tma, dims, real)
    ref = _c2r(tma, dims, spec)
    tma.vpfft_set_tma_passes(1)
    got = _c2r(tma, dims, spec)
    assert np.array_equal(got, ref)
    np.testing.assert_allclose(got, real, rtol=0, atol=3e-6 * np.abs(real).max())


def test_mixed_solve_same_bits(tma):
    n = 64
    R = fixtures.polycrystal(n, n, n, 40, 5)
    e = fixtures.edot_from_matrix(np.diag([1.0, 0.0, -1.0]))
    mat = vp.material(gamma_dot_base=1.0, rate_sensitivity=20, crss=1.0)
    out = {}
    for on in (0, 1):
        tma.vpfft_set_tma_passes(on)
        g = vp.MaterialGrid(n, n, n, material=mat, precision="mixed")
        g.SendDataAndInitialize(R)
        g.InitializeComputation(e)
        g.BuildLinearRefMediumStiffness()
        hist = g.FixedPoint(e, 8, 0.0)
        out[on] = (hist, g.Stress(), g.LagrangeMultiplier())
        g.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
