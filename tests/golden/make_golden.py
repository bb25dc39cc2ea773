"""Generate the golden fixtures of the parity tests from the reference itself.

    python tests/golden/make_golden.py [case ...]      (default: all small cases)

Each case builds a seeded synthetic microstructure with the product's host-side
fixture generator (vpfft_b200.fixtures.polycrystal: periodic Voronoi, uniform
SO(3) orientations), runs the reference's own MaterialGrid code compiled
against the single-process MPI/FFTW/Eigen stand-ins (oracle/_ref/vpfft_ref,
built by `make -C oracle ref`), and stores inputs and outputs in
tests/golden/<case>.npz.  The reference sources are only needed here, when the
fixtures are (re)generated; the tests read the committed .npz files.

Stored per case: the inputs (dims, material, strain rate, dt, eps, max_iter,
increments, voxel lengths, orientations or their SHA-256 for the large case),
per increment the iteration count, <sigma>, the per-iteration history
(<sigma>, <edot>, delta_sigma, delta_eps) and L0, and the fields after the run
(stress, Lagrange multiplier, orientation, CRSS, accumulated shear, P and d~ of
the last iteration; for the 64^3 case every field's mean and RMS after each
increment, and sampled voxels after increments 1, 5, 10, 15 and 20).
"""
from __future__ import annotations

import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refio  # noqa: E402
from vpfft_b200 import fixtures  # noqa: E402

S2, S6 = np.sqrt(2.0), np.sqrt(6.0)


def edot_of(L):
    return fixtures.edot_from_matrix(np.asarray(L, np.float64))


UNIAXIAL = np.diag([1.0, -0.5, -0.5])      # configs 1-2: uniaxial tension
PLANE_STRAIN = np.diag([1.0, 0.0, -1.0])   # config 3: plane-strain compression

# Voce constants of the 64^3 multi-increment config (tau0=1, tau1=0.5,
# theta0=20, theta1=1, hardening matrix all 1), also used by the small cases.
VOCE = dict(tau0=1.0, tau1=0.5, theta0=20.0, theta1=1.0, h=1.0)

CASES = {
    # config 1: 16^3, 8 grains, n=10, gdot0=1, tau=1, uniaxial, one increment
    "c1_16": dict(dims=(16, 16, 16), grains=8, seed=1, n=10, L=UNIAXIAL, nsteps=1, max_iter=100,
                  dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0), dump_iters=(0, 1, 2)),
    # hardening + texture over three increments
    "hard_16": dict(dims=(16, 16, 16), grains=12, seed=7, n=10, L=UNIAXIAL, nsteps=3,
                    max_iter=30, dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0), dump_iters=()),
    # non-cubic, odd and radix-3/5 dimensions, anisotropic voxels, plane strain
    "odd_15x12x10": dict(dims=(15, 12, 10), grains=6, seed=3, n=10, L=PLANE_STRAIN, nsteps=1,
                         max_iter=40, dt=0.005, eps=1e-5, h=(1.0, 1.5, 0.8), dump_iters=()),
    # the config-3 material (n=20, plane strain) on a small grid
    "n20_16": dict(dims=(16, 16, 16), grains=30, seed=11, n=20, L=PLANE_STRAIN, nsteps=1,
                   max_iter=50, dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0), dump_iters=()),
    # config 2: 64^3, 125 grains, 20 increments of uniaxial tension with Voce
    # hardening and texture update (long: tens of minutes on one core)
    "c2_64": dict(dims=(64, 64, 64), grains=125, seed=2, n=10, L=UNIAXIAL, nsteps=20,
                  max_iter=100, dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0), dump_iters=(),
                  sample=4096, sample_stride=4, store_increments=(0, 4, 9, 14, 19)),
}
SMALL = ["c1_16", "hard_16", "odd_15x12x10", "n20_16"]


def make_case(name: str, binary: str = refio.REF_BIN) -> str:
    c = CASES[name]
    nx, ny, nz = c["dims"]
    n = nx * ny * nz
    R = fixtures.polycrystal(nx, ny, nz, c["grains"], c["seed"])
    mat = refio.Material.uniform(1.0, c["n"], VOCE["tau0"], VOCE["tau1"], VOCE["theta0"],
                                 VOCE["theta1"], VOCE["h"])
    edot = edot_of(c["L"])
    case = refio.Case(c["dims"], R, np.zeros((n, 5)), np.ones(12), mat, edot, nsteps=c["nsteps"],
                      max_iter=c["max_iter"], dt=c["dt"], eps=c["eps"], h=c["h"])
    sample = c.get("sample")
    with tempfile.TemporaryDirectory() as td:
        out = refio.run(binary, case, td, dump_iters=c["dump_iters"],
                        dump_increments=sample is not None)
    hist = refio.iteration_history(out, c["dims"], edot)
    L0s = refio.l0_per_increment(out, nx)
    rec = dict(
        dims=np.array(c["dims"]), grains=np.array(c["grains"]), seed=np.array(c["seed"]),
        rate_sensitivity=np.array(c["n"]), gamma_dot_base=np.array(1.0), crss0=np.array(1.0),
        tau0=np.array(VOCE["tau0"]), tau1=np.array(VOCE["tau1"]), theta0=np.array(VOCE["theta0"]),
        theta1=np.array(VOCE["theta1"]), hardening=np.array(VOCE["h"]),
        velocity_gradient=np.asarray(c["L"]), edot=edot, nsteps=np.array(c["nsteps"]),
        max_iter=np.array(c["max_iter"]), dt=np.array(c["dt"]), eps=np.array(c["eps"]),
        h=np.array(c["h"]), iters=out["iters"], avg_stress=out["avg_stress"],
        hist_counts=np.array([len(h) for h in hist]),
        history=np.array([np.concatenate([s, e, [ds, de]]) for h in hist for (s, e, ds, de) in h]),
        L0=np.array(L0s), voxlen=out["voxlen"],
        R_in_sha256=np.array(hashlib.sha256(np.ascontiguousarray(R).tobytes()).hexdigest()),
        oracle=np.array(os.path.basename(binary)),
    )
    if sample is None:
        rec.update(R_in=R, sigma=out["sigma"], **{"lambda": out["lambda"]}, R=out["R"],
                   crss=out["crss"], accshear=out["accshear"], P_last=out["P_last"],
                   dtilde_last=out["dtilde_last"])
        for k in c["dump_iters"]:
            for f in ("sigma", "lambda", "P", "dtilde"):
                rec[f"it{k}_{f}"] = out[f"it{k}_{f}"]
    else:
        idx = np.unique(np.concatenate([np.arange(0, n, n // (sample // 2)),
                                        np.random.default_rng(0).choice(n, sample // 2, False)]))
        idx = idx[::c.get("sample_stride", 1)]
        rec["sample_index"] = idx
        for s in range(c["nsteps"]):
            for f in ("sigma", "lambda", "R", "crss"):
                full = out[f"inc{s}_{f}"]
                if s in c.get("store_increments", range(c["nsteps"])):
                    rec[f"inc{s}_{f}"] = full[idx]
                rec[f"inc{s}_{f}_mean"] = full.mean(axis=0)
                rec[f"inc{s}_{f}_rms"] = np.sqrt((full ** 2).mean(axis=0))
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **rec)
    return path


def main(argv):
    names = argv or SMALL
    for nm in names:
        p = make_case(nm)
        print(nm, "->", os.path.relpath(p, ROOT), f"{os.path.getsize(p) / 1e6:.2f} MB")


if __name__ == "__main__":
    main(sys.argv[1:])
