"""Synthetic microstructures and strain-rate helpers (host code of the C ABI;
no GPU needed).  See vpfft_b200/csrc/fixtures.cpp for the exact recipe."""
from __future__ import annotations

import numpy as np

from . import capi
from .capi import check, dptr, f64


def polycrystal(nx: int, ny: int, nz: int, n_grains: int, seed: int, with_grains: bool = False):
    """Periodic Voronoi polycrystal with uniform random orientations: (N, 9)."""
    n = nx * ny * nz
    R = np.zeros(n * 9)
    g = np.zeros(n, np.int32)
    check(capi.load().vpfft_fixture_polycrystal(nx, ny, nz, n_grains, seed, dptr(R),
                                                capi.iptr(g)))
    R = R.reshape(n, 9)
    return (R, g) if with_grains else R


def edot_from_matrix(L) -> np.ndarray:
    """EigenRep(SMatrix3x3) of a velocity gradient (LinearAlgebra.h:307-312)."""
    out = np.zeros(5)
    capi.load().vpfft_edot_from_matrix(dptr(f64(L, (9,))), dptr(out))
    return out


def matrix_from_edot(e) -> np.ndarray:
    """EigenRep::ToMatrixRep (LinearAlgebra.h:352-360): (3,3)."""
    out = np.zeros(9)
    capi.load().vpfft_matrix_from_edot(dptr(f64(e, (5,))), dptr(out))
    return out.reshape(3, 3)


def random_traceless_velocity_gradient(rng: np.random.Generator) -> np.ndarray:
    """Gaussian 3x3 with the trace removed from the symmetric part and scaled
    so that the equivalent strain rate sqrt(2/3 D:D) of D = sym(L) is 1."""
    L = rng.normal(size=(3, 3))
    L -= np.eye(3) * np.trace(L) / 3.0
    D = 0.5 * (L + L.T)
    eq = np.sqrt(2.0 / 3.0 * np.sum(D * D))
    return L / eq


def two_grain(nx: int, ny: int, nz: int) -> np.ndarray:
    """The config's TwoGrainInit microstructure (UnitTester::SetMaterialGrid,
    UnitTester.cpp:46-74): (N, 9)."""
    R = np.zeros((nx * ny * nz, 9))
    check(capi.load().vpfft_fixture_two_grain(nx, ny, nz, dptr(R)))
    return R


def euler_matrix(phi: float, theta: float, psi: float) -> np.ndarray:
    """SMatrix3x3::BuildActiveEulerMatrix (LinearAlgebra.cpp:160-181), radians: (3, 3)."""
    R = np.zeros(9)
    check(capi.load().vpfft_euler_matrix(float(phi), float(theta), float(psi), dptr(R)))
    return R.reshape(3, 3)
