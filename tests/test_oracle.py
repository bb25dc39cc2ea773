"""The oracle itself: the plain-C restatement against the reference's golden
fixtures (bit for bit), against the reference build when present, and its
building blocks against independent numpy computations.  CPU only."""
import os
import tempfile

import numpy as np
import pytest

from oracle import portlib, refio

SMALL = ["c1_16", "hard_16", "odd_15x12x10", "n20_16", "shear_16", "shear_24", "rich_n7",
         "n1_16"]


def case_from_golden(g):
    dims = tuple(int(x) for x in g["dims"])
    n = int(np.prod(dims))
    mat = refio.Material.uniform(float(g["gamma_dot_base"]), int(g["rate_sensitivity"]),
                                 float(g["tau0"]), float(g["tau1"]), float(g["theta0"]),
                                 float(g["theta1"]), float(g["hardening"]))
    crss = g["crss_in"] if "crss_in" in g else np.full(12, float(g["crss0"]))
    return refio.Case(dims, g["R_in"], np.zeros((n, 5)), crss, mat,
                      g["edot"], nsteps=int(g["nsteps"]), max_iter=int(g["max_iter"]),
                      dt=float(g["dt"]), eps=float(g["eps"]), h=tuple(g["h"]),
                      edot_steps=g.get("edot_steps"))


@pytest.mark.parametrize("name", SMALL)
def test_port_reproduces_reference_golden_bitwise(name, golden, port):
    g = golden(name)
    case = case_from_golden(g)
    dump = {"c1_16": (0, 1, 2), "shear_16": (0, 1)}.get(name, ())
    with tempfile.TemporaryDirectory() as td:
        out = refio.run(refio.PORT_BIN, case, td, dump_iters=dump)
    assert np.array_equal(out["iters"], g["iters"])
    assert np.array_equal(out["avg_stress"], g["avg_stress"])
    hist = refio.iteration_history(out, case.dims,
                                   case.edot if case.edot_steps is None else case.edot_steps)
    rows = np.array([np.concatenate([s, e, [a, b]]) for h in hist for (s, e, a, b) in h])
    assert np.array_equal(rows, g["history"])
    assert np.array_equal(np.array(refio.l0_per_increment(out, case.dims[0])), g["L0"])
    for k in ("sigma", "lambda", "R", "crss", "accshear", "P_last", "dtilde_last", "voxlen"):
        assert np.array_equal(out[k], g[k]), k
    for k in dump:
        for f in ("sigma", "lambda", "P", "dtilde"):
            assert np.array_equal(out[f"it{k}_{f}"], g[f"it{k}_{f}"]), (k, f)


@pytest.mark.skipif(not os.path.exists(refio.REF_BIN), reason="reference build not present")
def test_port_matches_reference_build_on_random_case(port):
    rng = np.random.default_rng(5)
    dims = (6, 10, 9)
    n = int(np.prod(dims))
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                  2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                  2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], axis=1)
    crss = rng.uniform(0.8, 1.3, size=(n, 12))
    mat = refio.Material.uniform(1.3, 7, 1.0, 0.5, 20.0, 1.0, 1.0)
    case = refio.Case(dims, R, np.zeros((n, 5)), crss, mat, np.array([0.3, -0.7, 0.2, 0.1, -0.4]),
                      nsteps=2, max_iter=12, dt=0.01, eps=1e-6, h=(1.0, 0.7, 1.2))
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        ra = refio.run(refio.REF_BIN, case, a, dump_iters=(1,))
        rb = refio.run(refio.PORT_BIN, case, b, dump_iters=(1,))
    for k in ("iters", "avg_stress", "allreduce", "sigma", "lambda", "R", "crss", "accshear",
              "P_last", "dtilde_last", "it1_P", "it1_dtilde"):
        assert np.array_equal(ra[k], rb[k]), k


@pytest.mark.skipif(not os.path.exists(refio.REF_BIN), reason="reference build not present")
def test_port_matches_reference_build_on_the_seed_sweep(port, lib):
    """The ten seeded 12^3 cases the device parity sweep (test_gpu_seeds.py)
    checks against the restatement: the restatement and the reference build
    agree bit for bit on each."""
    import concurrent.futures as cf

    from vpfft_b200 import fixtures

    dims = (12, 12, 12)
    n = int(np.prod(dims))
    edot = fixtures.edot_from_matrix(np.diag([1.0, -0.5, -0.5]))
    mat = refio.Material.uniform(1.0, 10, 1.0, 0.5, 20.0, 1.0)
    cases = {s: refio.Case(dims, fixtures.polycrystal(*dims, 8, s), np.zeros((n, 5)), np.ones(12),
                           mat, edot, nsteps=1, max_iter=100, dt=0.005, eps=1e-5)
             for s in range(1, 11)}
    with tempfile.TemporaryDirectory() as tmp, \
            cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        runs = {(s, b): ex.submit(refio.run, b, c, os.path.join(tmp, f"{s}_{i}"))
                for s, c in cases.items() for i, b in enumerate((refio.REF_BIN, refio.PORT_BIN))}
        out = {k: f.result() for k, f in runs.items()}
    for s in cases:
        ra, rb = out[(s, refio.REF_BIN)], out[(s, refio.PORT_BIN)]
        for k in ("iters", "avg_stress", "allreduce", "sigma", "lambda", "R", "crss", "accshear"):
            assert np.array_equal(ra[k], rb[k]), (s, k)


def test_dft_matches_numpy(port):
    rng = np.random.default_rng(1)
    for shape in [(8, 6, 5), (16, 12, 10), (3, 7, 4)]:
        a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        np.testing.assert_allclose(portlib.dft3d(a, -1), np.fft.fftn(a), rtol=0, atol=1e-12 * a.size)
        np.testing.assert_allclose(portlib.dft3d(a, +1), np.fft.ifftn(a) * a.size, rtol=0,
                                   atol=1e-12 * a.size)


def test_inverse5_matches_numpy(port):
    rng = np.random.default_rng(2)
    for _ in range(20):
        A = rng.normal(size=(5, 5)) + 3 * np.eye(5)
        np.testing.assert_allclose(portlib.inverse5(A), np.linalg.inv(A), rtol=1e-12, atol=1e-12)


def _basis():
    B = np.zeros((5, 3, 3))
    B[0] = np.diag([-1, 1, 0]) / np.sqrt(2)
    B[1] = np.diag([-1, -1, 2]) / np.sqrt(6)
    B[2][1, 2] = B[2][2, 1] = 1 / np.sqrt(2)
    B[3][0, 2] = B[3][2, 0] = 1 / np.sqrt(2)
    B[4][0, 1] = B[4][1, 0] = 1 / np.sqrt(2)
    return B


def test_green_matches_tensor_formula(port):
    """The restated Green operator equals an independent numpy evaluation of
    Gamma_ijkl = -k_j k_l [A k; k^T 0]^-1_ik projected on the basis."""
    rng = np.random.default_rng(3)
    B = _basis()
    M = rng.normal(size=(5, 5))
    L0 = M @ M.T + 5 * np.eye(5)
    Lt = np.einsum("ab,aij,bkl->ijkl", L0, B, B)
    for _ in range(10):
        k = rng.normal(size=3)
        k /= np.linalg.norm(k)
        A = np.einsum("j,l,ijkl->ik", k, k, Lt)
        Mb = np.zeros((4, 4))
        Mb[:3, :3] = A
        Mb[3, :3] = Mb[:3, 3] = k
        Ai = np.linalg.inv(Mb)[:3, :3]
        G4 = -np.einsum("j,l,ik->ijkl", k, k, Ai)
        G4s = (G4 + G4.transpose(1, 0, 2, 3) + G4.transpose(0, 1, 3, 2) + G4.transpose(1, 0, 3, 2)) / 4
        G = np.einsum("ijkl,aij,bkl->ab", G4s, B, B)
        np.testing.assert_allclose(portlib.green(L0, k), G, rtol=1e-10, atol=1e-12)


def test_schmid_basis_properties(port):
    """Crystal-frame Schmid tensors are traceless with |M|_F = 1/sqrt(2) and the
    sample-frame 5-vectors are their projections (identity orientation)."""
    m = portlib.schmid(np.eye(3).reshape(1, 9))[0]
    np.testing.assert_allclose(np.linalg.norm(m, axis=1), np.full(12, np.sqrt(0.5)), rtol=1e-14)
    # the 5-vector basis is orthonormal: projection preserves the inner product
    B = _basis()
    np.testing.assert_allclose(np.einsum("aij,bij->ab", B, B), np.eye(5), atol=1e-15)


def test_golden_inputs_reproducible(golden, lib):
    """The fixture generator reproduces the orientations stored in the goldens."""
    import hashlib

    from vpfft_b200 import fixtures

    for name in SMALL:
        g = golden(name)
        if int(g["grains"]) == 0:  # per-voxel random orientations, not a polycrystal
            continue
        dims = tuple(int(x) for x in g["dims"])
        R = fixtures.polycrystal(*dims, int(g["grains"]), int(g["seed"]))
        assert np.array_equal(R, g["R_in"]), name
        assert hashlib.sha256(R.tobytes()).hexdigest() == str(g["R_in_sha256"])


def test_oracle_polycrystal_equals_product_generator(port, lib):
    """The oracle-side generator (which lets the reference make its own
    benchmark inputs) gives the product's fixture bit for bit."""
    from vpfft_b200 import fixtures

    for dims, grains, seed in [((16, 16, 16), 8, 1), ((15, 12, 10), 6, 3), ((7, 5, 3), 40, 9),
                               ((33, 20, 17), 200, 5), ((1, 1, 1), 1, 0),
                               ((96, 64, 48), 1000, 2024)]:
        a, ga = portlib.polycrystal(*dims, grains, seed, threads=4, with_grains=True)
        b, gb = fixtures.polycrystal(*dims, grains, seed, with_grains=True)
        assert np.array_equal(a, b), dims
        assert np.array_equal(ga, gb), dims


@pytest.mark.skipif(not os.path.exists(refio.REF_BIN), reason="reference build not present")
def test_reference_as_several_ranks(port):
    """The reference run as P MPI ranks through the multi-process stand-ins
    (slab decomposition along x, uneven slabs and an empty rank included)
    agrees with the one-rank run: equal iteration counts, every reduced value
    within 1e-13 relative (only the order of the cross-rank sums differs), and
    the generated inputs equal explicit ones."""
    from vpfft_b200 import fixtures

    dims = (16, 12, 10)
    n = int(np.prod(dims))
    mat = refio.Material.uniform(1.0, 10, 1.0, 0.5, 20.0, 1.0)
    edot = fixtures.edot_from_matrix(np.diag([1.0, 0.0, -1.0]))
    gen = refio.Case(dims, None, None, np.ones(12), mat, edot, nsteps=2, max_iter=12, dt=0.005,
                     eps=1e-5)
    runs = {}
    with tempfile.TemporaryDirectory() as tmp:
        for ranks in (1, 2, 3, 5):
            runs[ranks] = refio.run(refio.REF_BIN, gen, os.path.join(tmp, str(ranks)),
                                    extra_args=["--generate", 7, 11, "--ranks", ranks,
                                                "--timing-only"])
        explicit = refio.Case(dims, portlib.polycrystal(*dims, 7, 11), np.zeros((n, 5)),
                              np.ones(12), mat, edot, nsteps=2, max_iter=12, dt=0.005, eps=1e-5)
        one = refio.run(refio.REF_BIN, explicit, os.path.join(tmp, "explicit"))
    assert np.array_equal(one["allreduce"], runs[1]["allreduce"])
    for ranks, out in runs.items():
        assert np.array_equal(out["iters"], one["iters"]), ranks
        scale = np.abs(one["allreduce"]).max()
        assert np.abs(out["allreduce"] - one["allreduce"]).max() <= 1e-13 * scale, ranks
        assert len(out["fwd_times"]) == len(one["fwd_times"])


def test_oracle_edot_projection_equals_product(lib):
    from vpfft_b200 import fixtures

    rng = np.random.default_rng(4)
    for L in [np.diag([1.0, 0.0, -1.0]), np.diag([1.0, -0.5, -0.5])] + \
            [fixtures.random_traceless_velocity_gradient(rng) for _ in range(5)]:
        assert np.array_equal(refio.edot_from_matrix(L), fixtures.edot_from_matrix(L))
