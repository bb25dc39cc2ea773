"""vpfft_solve_constrained_constitutive_noalloc against the allocating entry
point vpfft_solve_constrained_constitutive on the same inputs, two calls in a
row through the C ABI (the second smaller and with a different iteration cap,
so stale scratch contents or an uncleared counter would show).  Tolerance:
1e-13 relative per stress component (both run the same per-point solve)."""
import ctypes as C

import numpy as np
import pytest

from oracle import portlib
from vpfft_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _inputs(golden, n, seed):
    g = golden("c1_16")
    N = g["R_in"].shape[0]
    idx = np.random.default_rng(seed).choice(N, n, replace=False)
    m = np.ascontiguousarray(portlib.schmid(g["R_in"][idx]).reshape(n, 60))
    s0 = g["it0_sigma"][idx]
    mx = np.abs(np.einsum("nsc,nc->ns", m.reshape(n, 12, 5), s0)).max(axis=1)
    s0 = np.ascontiguousarray(s0 / mx[:, None])
    crss = np.ones((n, 12))
    lam = np.ascontiguousarray(g["it0_lambda"][idx])
    d = np.ascontiguousarray(g["it1_dtilde"][idx])
    L0 = np.ascontiguousarray(g["L0"][0].reshape(5, 5).T.ravel())  # column-major
    edot = np.ascontiguousarray(g["edot"], dtype=np.float64)
    return s0, m, crss, lam, d, L0, edot


def _call(lib, fn, args, n, max_iter, noalloc):
    s0, m, crss, lam, d, L0, edot = args
    mat = capi.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0)
    out, err = np.zeros((n, 5)), np.zeros(n)
    extra = []
    cnt = C.c_int64(-1)
    if noalloc:
        extra = [C.byref(cnt)]
    st = fn(n, capi.dptr(s0), capi.dptr(m), capi.dptr(crss), C.byref(mat), capi.dptr(edot),
            capi.dptr(lam), capi.dptr(d), capi.dptr(L0), 5e-4, 1e9, max_iter, capi.dptr(out),
            capi.dptr(err), *extra)
    capi.check(st)
    return out, err, cnt.value


def test_noalloc_matches_allocating_entry_point_twice(lib, golden):
    cases = [(capi.NOALLOC_MAX_POINTS, 100, 11), (777, 2, 12)]
    for n, max_iter, seed in cases:
        args = _inputs(golden, n, seed)
        ref, ref_err, _ = _call(lib, lib.vpfft_solve_constrained_constitutive, args, n, max_iter,
                                False)
        got, got_err, cnt = _call(lib, lib.vpfft_solve_constrained_constitutive_noalloc, args, n,
                                  max_iter, True)
        rel = np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)
        assert rel.max() <= TOL, (n, rel.max())
        np.testing.assert_allclose(got_err, ref_err, rtol=TOL, atol=0)
        assert cnt == int(np.count_nonzero(~(ref_err < 5e-4))), (n, cnt)
    # the capped second call really left points unconverged, so the count was exercised
    assert cnt > 0


def test_noalloc_second_call_allocates_nothing(lib, golden):
    """After the set-up call, a call leaves the device's free memory exactly as
    it was (cudaMemGetInfo through torch, which shares the primary context)."""
    import torch

    torch.cuda.init()
    torch.cuda.mem_get_info(0)
    n = 1024
    args = _inputs(golden, n, 21)
    _call(lib, lib.vpfft_solve_constrained_constitutive_noalloc, args, n, 100, True)  # set-up
    free0, _ = torch.cuda.mem_get_info(0)
    out, _, _ = _call(lib, lib.vpfft_solve_constrained_constitutive_noalloc, args, n, 100, True)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert np.all(np.isfinite(out))


def test_noalloc_refuses_oversize_batch(lib, golden):
    n = capi.NOALLOC_MAX_POINTS + 1
    z5, z60, z12 = np.zeros((n, 5)), np.zeros((n, 60)), np.zeros((n, 12))
    mat = capi.material()
    st = lib.vpfft_solve_constrained_constitutive_noalloc(
        n, capi.dptr(z5), capi.dptr(z60), capi.dptr(z12), C.byref(mat), capi.dptr(np.zeros(5)),
        capi.dptr(z5), capi.dptr(z5), capi.dptr(np.eye(5).ravel().copy()), 5e-4, 1e9, 100,
        capi.dptr(z5), None, None)
    assert st == capi.ERR_UNSUPPORTED_SIZE
    assert b"scratch" in lib.vpfft_last_error(None)
