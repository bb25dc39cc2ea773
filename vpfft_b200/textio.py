"""The reference's text formats over the C ABI (host only): the Print* field
dumps of MaterialGrid (MaterialGrid.cpp:15-100), WriteRandomMaterial /
ReadRandomMaterial (UnitTester.cpp:116-167) and the Euler-angle texture reader
ReadRicardoData (UnitTester.cpp:237-265)."""
from __future__ import annotations

import numpy as np

from . import capi
from .capi import check, dptr, f64

_KINDS = {"strain": capi.PRINT_STRAIN, "stress": capi.PRINT_STRESS,
          "lagrange": capi.PRINT_LAGRANGE, "polarization": capi.PRINT_POLARIZATION}


def print_field(path: str, kind: str, dims, re, im=None) -> None:
    nx, ny, nz = dims
    n = nx * ny * nz
    r = f64(re, (n, 5))
    i = None if im is None else f64(im, (n, 5))
    check(capi.load().vpfft_print_field(str(path).encode(), _KINDS[kind], nx, ny, nz, dptr(r),
                                        dptr(i) if i is not None else None))


def WriteRandomMaterial(path: str, dims, Orientations, Stress) -> None:
    nx, ny, nz = dims
    n = nx * ny * nz
    check(capi.load().vpfft_write_random_material(str(path).encode(), nx, ny, nz,
                                                  dptr(f64(Orientations, (n, 9))),
                                                  dptr(f64(Stress, (n, 5)))))


def ReadRandomMaterial(path: str, dims):
    """Returns (orientations (N, 9), stress (N, 5))."""
    nx, ny, nz = dims
    n = nx * ny * nz
    R, S = np.zeros((n, 9)), np.zeros((n, 5))
    check(capi.load().vpfft_read_random_material(str(path).encode(), nx, ny, nz, dptr(R),
                                                 dptr(S)))
    return R, S


def ReadRicardoData(path: str, dims, Orientations=None) -> np.ndarray:
    """Orientations (N, 9) from an Euler-angle texture file; voxels not listed
    keep the values of `Orientations` (identity by default)."""
    nx, ny, nz = dims
    n = nx * ny * nz
    R = (np.tile(np.eye(3).ravel(), (n, 1)) if Orientations is None
         else f64(Orientations, (n, 9)).copy())
    check(capi.load().vpfft_read_euler_texture(str(path).encode(), nx, ny, nz, dptr(R)))
    return R
