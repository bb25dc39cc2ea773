"""Generate the golden fixtures of the parity tests from the reference itself.

    python tests/golden/make_golden.py [case ...]      (default: all small cases)

Each case builds a seeded synthetic microstructure with the product's host-side
fixture generator (vpfft_b200.fixtures.polycrystal: periodic Voronoi, uniform
SO(3) orientations), runs the reference's own MaterialGrid code compiled
against the single-process MPI/FFTW/Eigen stand-ins (oracle/_ref/vpfft_ref,
built by `make -C oracle ref REF_SRC=<reference Src>`), and stores inputs and outputs in
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
# Input classes of the batched and serving workloads and of the solver's less
# common paths, each against the reference build:
CASES.update({
    # random traceless velocity gradients (Gaussian entries, symmetric part
    # scaled to equivalent strain rate 1), a different one per increment, as
    # the serving workload applies to a persistent RVE; Voce + texture between
    "shear_16": dict(dims=(16, 16, 16), grains=20, seed=21, n=10, L_seed=101, nsteps=2,
                     max_iter=100, dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0), dump_iters=(0, 1)),
    # the same recipe on an edge that takes the runtime-plan FFT engine (24)
    "shear_24": dict(dims=(24, 24, 24), grains=40, seed=23, n=10, L_seed=103, nsteps=1,
                     max_iter=100, dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0), dump_iters=()),
    # a rate exponent with no compile-time kernel (n = 7), per-voxel random
    # orientations and CRSS, gdot0 = 1.3, a full 5-component strain rate,
    # anisotropic voxels, two increments
    "rich_n7": dict(dims=(12, 10, 9), orient="random", orient_seed=5, crss="random", gdot=1.3,
                    n=7, edot=(0.3, -0.7, 0.2, 0.1, -0.4), nsteps=2, max_iter=30, dt=0.01,
                    eps=1e-6, h=(1.0, 0.7, 1.2), dump_iters=()),
    # the linear (n = 1) branch of the constitutive law (Solvers.cpp:177-180)
    "n1_16": dict(dims=(16, 16, 16), grains=8, seed=31, n=1, L=UNIAXIAL, nsteps=1, max_iter=50,
                  dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0), dump_iters=()),
})
SMALL = ["c1_16", "hard_16", "odd_15x12x10", "n20_16", "shear_16", "shear_24", "rich_n7",
         "n1_16"]

# RunVPFFT (MaterialGrid.cpp:1202-1228) itself, for its Stress_Strain.txt
STRESS_STRAIN = dict(dims=(16, 16, 16), grains=8, seed=1, n=10, L=UNIAXIAL, nsteps=3,
                     max_iter=30, dt=0.005, eps=1e-5, h=(1.0, 1.0, 1.0))


def random_orientations(n: int, seed: int) -> np.ndarray:
    """Per-voxel uniform random rotations (normalised Gaussian quaternions),
    row-major 3x3: (n, 9)."""
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                     2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                     2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], axis=1)


def case_inputs(c: dict):
    """(R, crss, material, edot, edot_steps, velocity gradients) of a case."""
    nx, ny, nz = c["dims"]
    n = nx * ny * nz
    if c.get("orient") == "random":
        R = random_orientations(n, c["orient_seed"])
    else:
        R = fixtures.polycrystal(nx, ny, nz, c["grains"], c["seed"])
    if c.get("crss") == "random":
        crss = np.random.default_rng(c["orient_seed"] + 1).uniform(0.8, 1.3, size=(n, 12))
    else:
        crss = np.ones(12)
    mat = refio.Material.uniform(c.get("gdot", 1.0), c["n"], VOCE["tau0"], VOCE["tau1"],
                                 VOCE["theta0"], VOCE["theta1"], VOCE["h"])
    edot_steps, Ls = None, None
    if "L_seed" in c:
        rng = np.random.default_rng(c["L_seed"])
        Ls = np.array([fixtures.random_traceless_velocity_gradient(rng)
                       for _ in range(c["nsteps"])])
        edot_steps = np.array([edot_of(L) for L in Ls])
        edot = edot_steps[0]
    elif "edot" in c:
        edot = np.array(c["edot"], np.float64)
    else:
        Ls = np.asarray(c["L"])[None]
        edot = edot_of(c["L"])
    return R, crss, mat, edot, edot_steps, Ls


def make_case(name: str, binary: str = refio.REF_BIN) -> str:
    c = CASES[name]
    nx, ny, nz = c["dims"]
    n = nx * ny * nz
    R, crss, mat, edot, edot_steps, Ls = case_inputs(c)
    case = refio.Case(c["dims"], R, np.zeros((n, 5)), crss, mat, edot, nsteps=c["nsteps"],
                      max_iter=c["max_iter"], dt=c["dt"], eps=c["eps"], h=c["h"],
                      edot_steps=edot_steps)
    sample = c.get("sample")
    with tempfile.TemporaryDirectory() as td:
        out = refio.run(binary, case, td, dump_iters=c["dump_iters"],
                        dump_increments=sample is not None)
    hist = refio.iteration_history(out, c["dims"], edot if edot_steps is None else edot_steps)
    L0s = refio.l0_per_increment(out, nx)
    rec = dict(
        dims=np.array(c["dims"]), grains=np.array(c.get("grains", 0)),
        seed=np.array(c.get("seed", c.get("orient_seed", 0))),
        rate_sensitivity=np.array(c["n"]), gamma_dot_base=np.array(c.get("gdot", 1.0)),
        crss0=np.array(1.0),
        tau0=np.array(VOCE["tau0"]), tau1=np.array(VOCE["tau1"]), theta0=np.array(VOCE["theta0"]),
        theta1=np.array(VOCE["theta1"]), hardening=np.array(VOCE["h"]),
        velocity_gradient=np.zeros((0, 3, 3)) if Ls is None else Ls, edot=edot,
        nsteps=np.array(c["nsteps"]),
        max_iter=np.array(c["max_iter"]), dt=np.array(c["dt"]), eps=np.array(c["eps"]),
        h=np.array(c["h"]), iters=out["iters"], avg_stress=out["avg_stress"],
        hist_counts=np.array([len(h) for h in hist]),
        history=np.array([np.concatenate([s, e, [ds, de]]) for h in hist for (s, e, ds, de) in h]),
        L0=np.array(L0s), voxlen=out["voxlen"],
        R_in_sha256=np.array(hashlib.sha256(np.ascontiguousarray(R).tobytes()).hexdigest()),
        oracle=np.array(os.path.basename(binary)),
    )
    if edot_steps is not None:
        rec["edot_steps"] = edot_steps
    if np.asarray(crss).ndim == 2:
        rec["crss_in"] = crss
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


def make_stress_strain(binary: str = refio.REF_BIN) -> str:
    """Stress_Strain.txt written by the reference's RunVPFFT, and its inputs."""
    c = STRESS_STRAIN
    nx, ny, nz = c["dims"]
    n = nx * ny * nz
    R, crss, mat, edot, _, _ = case_inputs(c)
    case = refio.Case(c["dims"], R, np.zeros((n, 5)), crss, mat, edot, nsteps=c["nsteps"],
                      max_iter=c["max_iter"], dt=c["dt"], eps=c["eps"], h=c["h"])
    with tempfile.TemporaryDirectory() as td:
        refio.run(binary, case, td, run_vpfft=True)
        with open(os.path.join(td, "Stress_Strain.txt"), "rb") as fh:
            text = fh.read()
    path = os.path.join(HERE, "io", "stress_strain_16.txt")
    with open(path, "wb") as fh:
        fh.write(text)
    return path


def main(argv):
    names = argv or SMALL + ["stress_strain"]
    for nm in names:
        if nm == "stress_strain":
            p = make_stress_strain()
            print(nm, "->", os.path.relpath(p, ROOT))
            continue
        p = make_case(nm)
        print(nm, "->", os.path.relpath(p, ROOT), f"{os.path.getsize(p) / 1e6:.2f} MB")


if __name__ == "__main__":
    main(sys.argv[1:])
