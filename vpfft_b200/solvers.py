"""Batched device versions of VPFFT::Solvers (Solvers.h:51-153).

Each function takes numpy arrays for n voxels and runs the same device code
the grid kernels use.  Arrays: stress (n,5), schmid (n,12,5), crss (n,12),
L0 5x5 indexed [i, j].
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import check, dptr, f64


def _mat(m):
    return C.byref(m if m is not None else capi.material())


def _l0_colmajor(L0) -> np.ndarray:
    return f64(np.asarray(L0, np.float64).T, (25,))


def SolveConstitutiveEquations(InitialStressState, SchmidtTensors, CRSS, material, StrainRate,
                               EpsilonConvergence=5e-4, MaxResolvedStress=2.0,
                               MaxNumIterations=1000) -> np.ndarray:
    """Solvers::SolveConstitutiveEquations (Solvers.cpp:19-101)."""
    s0 = f64(InitialStressState).reshape(-1, 5)
    n = s0.shape[0]
    sch, cr = f64(SchmidtTensors, (n, 60)), f64(CRSS, (n, 12))
    out = np.zeros((n, 5))
    lib = capi.load()
    check(lib.vpfft_solve_constitutive(n, dptr(s0), dptr(sch), dptr(cr), _mat(material),
                                       dptr(f64(StrainRate, (5,))), EpsilonConvergence,
                                       MaxResolvedStress, int(MaxNumIterations), dptr(out)))
    return out


def SolveConstrainedConstitutiveEquations(InitialStressState, SchmidtTensors, CRSS, material,
                                          MacroscopicStrainRate, LagrangeMultiplier,
                                          LocalDisplacementVariation, HomogeonousReference,
                                          EpsilonConvergence=5e-4, MaxResolvedStress=1e9,
                                          MaxNumIterations=100):
    """Solvers::SolveConstrainedConstitutiveEquations (Solvers.cpp:111-222).
    Returns (stress (n,5), NR_Error_Out (n,))."""
    s0 = f64(InitialStressState).reshape(-1, 5)
    n = s0.shape[0]
    sch, cr = f64(SchmidtTensors, (n, 60)), f64(CRSS, (n, 12))
    lam, d = f64(LagrangeMultiplier, (n, 5)), f64(LocalDisplacementVariation, (n, 5))
    out, err = np.zeros((n, 5)), np.zeros(n)
    lib = capi.load()
    check(lib.vpfft_solve_constrained_constitutive(
        n, dptr(s0), dptr(sch), dptr(cr), _mat(material), dptr(f64(MacroscopicStrainRate, (5,))),
        dptr(lam), dptr(d), dptr(_l0_colmajor(HomogeonousReference)), EpsilonConvergence,
        MaxResolvedStress, int(MaxNumIterations), dptr(out), dptr(err)))
    return out, err


def ApplyConstitutiveEquations(StressState, SchmidtTensors, CRSS, material) -> np.ndarray:
    """Solvers::ApplyConstitutiveEquations (Solvers.cpp:255-274)."""
    s = f64(StressState).reshape(-1, 5)
    n = s.shape[0]
    out = np.zeros((n, 5))
    check(capi.load().vpfft_apply_constitutive(n, dptr(s), dptr(f64(SchmidtTensors, (n, 60))),
                                               dptr(f64(CRSS, (n, 12))), _mat(material),
                                               dptr(out)))
    return out


def SolveSachEquation(SchmidtTensors, CRSS, StrainRate) -> np.ndarray:
    """Solvers::SolveSachEquation (Solvers.cpp:230-243)."""
    sch = f64(SchmidtTensors).reshape(-1, 60)
    n = sch.shape[0]
    out = np.zeros((n, 5))
    check(capi.load().vpfft_solve_sachs(n, dptr(sch), dptr(f64(CRSS, (n, 12))),
                                        dptr(f64(StrainRate, (5,))), dptr(out)))
    return out


def SchmidtTensors(Orientations) -> np.ndarray:
    """UpdateSchmidtTensors for n orientations (MaterialGrid.cpp:107-124): (n,12,5)."""
    R = f64(Orientations).reshape(-1, 9)
    n = R.shape[0]
    out = np.zeros((n, 60))
    check(capi.load().vpfft_schmid_tensors(n, dptr(R), dptr(out)))
    return out.reshape(n, 12, 5)


def GreenApply(k_index, dims, h, L0, phat, precision: str = "fp64") -> np.ndarray:
    """d^ = -Gbar(k) P^ at integer wave-vector indices k_index (n,3); phat (n,5) complex."""
    k = np.ascontiguousarray(k_index, np.int32).reshape(-1, 3)
    n = k.shape[0]
    p = np.ascontiguousarray(np.asarray(phat, np.complex128).reshape(n, 5)).view(np.float64)
    out = np.zeros((n, 10))
    prec = capi.PREC_FP64 if precision == "fp64" else capi.PREC_MIXED
    check(capi.load().vpfft_green_apply(n, k.ctypes.data_as(C.POINTER(C.c_int32)), dims[0],
                                        dims[1], dims[2], dptr(f64(h, (3,))),
                                        dptr(_l0_colmajor(L0)), dptr(f64(p, (n * 10,))),
                                        dptr(out), prec))
    return out.view(np.complex128).reshape(n, 5)


def fft3d_r2c(real, dims, precision: str = "fp64") -> np.ndarray:
    """Forward (unnormalised) device transform of real (ncomp, nx, ny, nz)."""
    nx, ny, nz = dims
    a = f64(real).reshape(-1, nx * ny * nz)
    nc = a.shape[0]
    nh = nz // 2 + 1
    out = np.zeros(nc * nx * ny * nh * 2)
    prec = capi.PREC_FP64 if precision == "fp64" else capi.PREC_MIXED
    check(capi.load().vpfft_fft3d_r2c(nx, ny, nz, nc, dptr(f64(a, (-1,))), dptr(out), prec))
    return out.view(np.complex128).reshape(nc, nx, ny, nh)


def fft3d_c2r(spec, dims, precision: str = "fp64") -> np.ndarray:
    """Inverse device transform (divides by N) of a half spectrum (ncomp, nx, ny, nz/2+1)."""
    nx, ny, nz = dims
    s = np.ascontiguousarray(np.asarray(spec, np.complex128)).reshape(-1, nx, ny, nz // 2 + 1)
    nc = s.shape[0]
    out = np.zeros(nc * nx * ny * nz)
    prec = capi.PREC_FP64 if precision == "fp64" else capi.PREC_MIXED
    check(capi.load().vpfft_fft3d_c2r(nx, ny, nz, nc, dptr(f64(s.view(np.float64), (-1,))),
                                      dptr(out), prec))
    return out.reshape(nc, nx, ny, nz)
