"""ctypes access to the per-voxel routines of the plain-C restatement
(oracle/_build/liboracle.so, built by `make -C oracle port`).

Test-oracle infrastructure: used only by tests/ and __graft_entry__.smoke()
as the checker of the device kernels.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

_D = C.POINTER(C.c_double)


class OracleMaterial(C.Structure):
    _fields_ = [
        ("gamma_dot_base", C.c_double * 12),
        ("rate_sensitivity", C.c_int * 12),
        ("tau0", C.c_double * 12),
        ("tau1", C.c_double * 12),
        ("theta0", C.c_double * 12),
        ("theta1", C.c_double * 12),
        ("hardening", C.c_double * 144),
    ]


def build() -> None:
    """Compile the restatement (and its CLI) if needed; needs gcc and make."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True, capture_output=True)


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.oracle_schmid_sample.argtypes = [_D, _D]
        lib.oracle_sachs.argtypes = [_D, _D, _D, _D]
        lib.oracle_max_rss.argtypes = [_D, _D, _D]
        lib.oracle_max_rss.restype = C.c_double
        lib.oracle_solve_unconstrained.argtypes = [_D, _D, _D, C.POINTER(OracleMaterial), _D,
                                                   C.c_double, C.c_double, C.c_int, _D]
        lib.oracle_solve_constrained.argtypes = [_D, _D, _D, C.POINTER(OracleMaterial), _D, _D, _D,
                                                 _D, C.c_double, C.c_double, C.c_int, _D, _D]
        lib.oracle_apply_constitutive.argtypes = [_D, _D, _D, C.POINTER(OracleMaterial), _D]
        lib.oracle_green.argtypes = [_D, _D, _D]
        lib.oracle_inverse5.argtypes = [_D, _D]
        lib.oracle_dft3d_inplace.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t,
                                             C.c_int]
        lib.oracle_polycrystal.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                           _D, C.POINTER(C.c_int32)]
        lib.oracle_polycrystal.restype = C.c_int
        _lib = lib
    return _lib


def _p(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(_D)


def material(gdot=1.0, n=10, tau0=1.0, tau1=0.5, theta0=20.0, theta1=1.0, h=1.0):
    m = OracleMaterial()
    m.gamma_dot_base[:] = [float(gdot)] * 12
    m.rate_sensitivity[:] = [int(n)] * 12
    m.tau0[:] = [float(tau0)] * 12
    m.tau1[:] = [float(tau1)] * 12
    m.theta0[:] = [float(theta0)] * 12
    m.theta1[:] = [float(theta1)] * 12
    m.hardening[:] = [float(h)] * 144
    return m


def schmid(R) -> np.ndarray:
    R = np.ascontiguousarray(R, np.float64).reshape(-1, 9)
    out = np.zeros((R.shape[0], 60))
    lib = load()
    for i in range(R.shape[0]):
        lib.oracle_schmid_sample(_p(R[i]), out[i].ctypes.data_as(_D))
    return out.reshape(-1, 12, 5)


def _col(L0):
    return np.ascontiguousarray(np.asarray(L0, np.float64).T).reshape(25)


def solve_constrained(s0, m, crss, mat, edot, lam, d, L0, eps=5e-4, max_rss=1e9, max_iter=100):
    lib = load()
    n = len(s0)
    out = np.zeros((n, 5))
    err = np.zeros(n)
    L = _col(L0)
    e = np.ascontiguousarray(edot, np.float64)
    for i in range(n):
        o = np.zeros(5)
        r = C.c_double()
        lib.oracle_solve_constrained(_p(s0[i]), _p(m[i]), _p(crss[i]), C.byref(mat), _p(e),
                                     _p(lam[i]), _p(d[i]), _p(L), eps, max_rss, max_iter,
                                     o.ctypes.data_as(_D), C.byref(r))
        out[i] = o
        err[i] = r.value
    return out, err


def solve_unconstrained(s0, m, crss, mat, edot, eps=5e-4, max_rss=2.0, max_iter=1000):
    lib = load()
    n = len(s0)
    out = np.zeros((n, 5))
    e = np.ascontiguousarray(edot, np.float64)
    for i in range(n):
        o = np.zeros(5)
        lib.oracle_solve_unconstrained(_p(s0[i]), _p(m[i]), _p(crss[i]), C.byref(mat), _p(e), eps,
                                       max_rss, max_iter, o.ctypes.data_as(_D))
        out[i] = o
    return out


def apply_constitutive(s, m, crss, mat):
    lib = load()
    out = np.zeros((len(s), 5))
    for i in range(len(s)):
        o = np.zeros(5)
        lib.oracle_apply_constitutive(_p(s[i]), _p(m[i]), _p(crss[i]), C.byref(mat),
                                      o.ctypes.data_as(_D))
        out[i] = o
    return out


def sachs(m, crss, edot):
    lib = load()
    out = np.zeros((len(m), 5))
    for i in range(len(m)):
        o = np.zeros(5)
        lib.oracle_sachs(_p(m[i]), _p(crss[i]), _p(edot), o.ctypes.data_as(_D))
        out[i] = o
    return out


def green(L0, k) -> np.ndarray:
    """Symmetrised projected Green operator (5x5 [i, j]) at unit wave vector k."""
    lib = load()
    G = np.zeros(25)
    lib.oracle_green(_p(_col(L0)), _p(k), G.ctypes.data_as(_D))
    return G.reshape(5, 5).T.copy()


def inverse5(A) -> np.ndarray:
    lib = load()
    out = np.zeros(25)
    lib.oracle_inverse5(_p(_col(A)), out.ctypes.data_as(_D))
    return out.reshape(5, 5).T.copy()


def dft3d(a: np.ndarray, sign: int) -> np.ndarray:
    """In-place-style unnormalised 3D DFT of a complex array (copy returned)."""
    x = np.ascontiguousarray(a, np.complex128).copy()
    nx, ny, nz = x.shape
    load().oracle_dft3d_inplace(x.ctypes.data, nx, ny, nz, sign)
    return x


def green_bar_dhat(L0, idx, dims, h, phat) -> np.ndarray:
    """The reference's effective operator on the Hermitian half spectrum:
    dhat = -(Op(k) + Op(-k))/2 phat with Op the Green operator, or inverse(-L0)
    on the Nyquist planes of even axes (MaterialGrid.cpp:690-740)."""
    nx, ny, nz = dims
    ix, iy, iz = idx
    if ix == 0 and iy == 0 and iz == 0:
        return np.zeros(5, complex)

    def ov(i, n):
        return n % 2 == 0 and (i == n // 2 or i == n // 2 + 1)

    def op(i3):
        jx, jy, jz = i3
        if ov(jx, nx) or ov(jy, ny) or ov(jz, nz):
            return inverse5(-np.asarray(L0))
        w = np.array([jx - nx if jx > nx // 2 else jx, jy - ny if jy > ny // 2 else jy,
                      jz - nz if jz > nz // 2 else jz], float)
        w = w / (np.array(dims, float) * np.asarray(h, float))
        w = w / np.linalg.norm(w)
        return green(L0, w)

    G = 0.5 * (op((ix, iy, iz)) + op(((nx - ix) % nx, (ny - iy) % ny, (nz - iz) % nz)))
    return -G @ np.asarray(phat)


def polycrystal(nx: int, ny: int, nz: int, grains: int, seed: int, threads: int = 1,
                with_grains: bool = False):
    """The oracle-side synthetic polycrystal (oracle/common/polycrystal.c):
    (N, 9) row-major orientations, and the grain of every voxel on request."""
    n = nx * ny * nz
    R = np.zeros((n, 9))
    g = np.zeros(n, np.int32)
    rc = load().oracle_polycrystal(nx, ny, nz, grains, seed, threads,
                                   R.ctypes.data_as(_D), g.ctypes.data_as(C.POINTER(C.c_int32)))
    if rc != 0:
        raise ValueError(f"oracle_polycrystal failed ({rc})")
    return (R, g) if with_grains else R
