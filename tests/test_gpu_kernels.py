"""Device building blocks against the oracle's restatement of the reference
routines (FP64 unless stated).  Tolerances are written per test."""
import numpy as np
import pytest

from oracle import portlib
from vpfft_b200 import capi, solvers

pytestmark = pytest.mark.gpu


def rand_rotations(rng, n, skew=0.0):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                  2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                  2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], axis=1)
    return R + skew * rng.normal(size=R.shape)


def test_schmid_tensors(lib, port):
    rng = np.random.default_rng(0)
    for skew in (0.0, 0.05):  # non-orthogonal R occurs after the additive texture update
        R = rand_rotations(rng, 200, skew)
        np.testing.assert_allclose(solvers.SchmidtTensors(R), portlib.schmid(R), rtol=0, atol=1e-14)


def _voxel_setup(golden, n=300):
    g = golden("c1_16")
    N = g["R_in"].shape[0]
    idx = np.random.default_rng(1).choice(N, n, replace=False)
    R = g["R_in"][idx]
    m = portlib.schmid(R)
    return g, idx, m


def test_sachs_and_apply(lib, port, golden):
    g, idx, m = _voxel_setup(golden)
    crss = np.ones((len(idx), 12))
    mat_o = portlib.material(1.0, 10)
    mat_d = capi.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0)
    e = g["edot"]
    np.testing.assert_allclose(solvers.SolveSachEquation(m, crss, e), portlib.sachs(m, crss, e),
                               rtol=1e-14, atol=1e-14)
    s = g["it1_sigma"][idx]
    d = solvers.ApplyConstitutiveEquations(s, m, crss, mat_d)
    o = portlib.apply_constitutive(s, m, crss, mat_o)
    np.testing.assert_allclose(d, o, rtol=1e-12, atol=1e-13 * np.abs(o).max())


def test_unconstrained_nr(lib, port, golden):
    g, idx, m = _voxel_setup(golden)
    crss = np.ones((len(idx), 12))
    e = g["edot"]
    s0 = portlib.sachs(m, crss, e)
    s0 /= np.maximum(1.0, np.abs(np.einsum("nsc,nc->ns", m, s0)).max(axis=1))[:, None]
    mat_o = portlib.material(1.0, 10)
    mat_d = capi.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0)
    o = portlib.solve_unconstrained(s0, m, crss, mat_o, e, 5e-4, 2.08, 1000)
    d = solvers.SolveConstitutiveEquations(s0, m, crss, mat_d, e, 5e-4, 2.08, 1000)
    rel = np.linalg.norm(d - o, axis=1) / np.linalg.norm(o, axis=1)
    assert rel.max() < 1e-10, rel.max()


def test_constrained_nr_on_reference_state(lib, port, golden):
    """One NR solve per voxel fed with the reference's iteration-1 inputs."""
    g, idx, m = _voxel_setup(golden)
    crss = np.ones((len(idx), 12))
    L0 = g["L0"][0]
    s0 = g["it0_sigma"][idx]
    mx = np.abs(np.einsum("nsc,nc->ns", m, s0)).max(axis=1)
    s0 = s0 / mx[:, None]
    lam = g["it0_lambda"][idx]
    d = g["it1_dtilde"][idx]
    mat_o = portlib.material(1.0, 10)
    mat_d = capi.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0)
    o, oe = portlib.solve_constrained(s0, m, crss, mat_o, g["edot"], lam, d, L0)
    dd, de = solvers.SolveConstrainedConstitutiveEquations(s0, m, crss, mat_d, g["edot"], lam, d, L0)
    rel = np.linalg.norm(dd - o, axis=1) / np.linalg.norm(o, axis=1)
    assert rel.max() < 1e-10, rel.max()
    # the reference's own NR result for these voxels (golden, sample-frame Schmid)
    ref = g["it1_sigma"][idx]
    rel2 = np.linalg.norm(dd - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert rel2.max() < 1e-10, rel2.max()


@pytest.mark.parametrize("dims,h", [((8, 6, 10), (1.0, 1.0, 1.0)), ((9, 8, 5), (1.0, 1.3, 0.7)),
                                    ((16, 16, 16), (1.0, 1.0, 1.0))])
def test_green_operator(lib, port, dims, h):
    """Gbar(k) on the half spectrum incl. the Nyquist-plane override and the
    k/-k average; FP64 <= 1e-12 relative, FP32 <= 2e-5 relative."""
    rng = np.random.default_rng(4)
    M = rng.normal(size=(5, 5))
    L0 = M @ M.T + 4 * np.eye(5)
    nx, ny, nz = dims
    ks = [(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz // 2 + 1)]
    ks = [ks[i] for i in rng.choice(len(ks), min(300, len(ks)), replace=False)] + [(0, 0, 0)]
    ph = rng.normal(size=(len(ks), 5)) + 1j * rng.normal(size=(len(ks), 5))
    ref = np.array([portlib.green_bar_dhat(L0, k, dims, h, p) for k, p in zip(ks, ph)])
    for prec, tol in (("fp64", 1e-12), ("mixed", 2e-5)):
        got = solvers.GreenApply(np.array(ks), dims, h, L0, ph, prec)
        err = np.abs(got - ref).max(axis=1) / (np.abs(ref).max(axis=1) + 1e-300)
        err[np.abs(ref).max(axis=1) == 0] = np.abs(got[np.abs(ref).max(axis=1) == 0]).max(initial=0)
        assert err.max() < tol, (prec, err.max())


@pytest.mark.parametrize("dims", [(16, 16, 16), (15, 12, 10), (8, 6, 5), (32, 24, 48), (5, 9, 15),
                                  (64, 64, 64), (1, 4, 3), (2, 2, 2), (96, 16, 128),
                                  (16, 256, 32), (48, 32, 512), (8, 384, 16), (192, 10, 16)])
def test_fft_r2c_and_c2r(lib, dims):
    rng = np.random.default_rng(6)
    a = rng.normal(size=(3,) + dims)
    ref = np.fft.rfftn(a, axes=(1, 2, 3))
    for prec, tol in (("fp64", 1e-12), ("mixed", 3e-6)):
        spec = solvers.fft3d_r2c(a, dims, prec)
        scale = np.abs(ref).max()
        assert np.abs(spec - ref).max() / scale < tol, prec
        back = solvers.fft3d_c2r(ref, dims, prec)
        assert np.abs(back - a).max() / np.abs(a).max() < tol, prec
